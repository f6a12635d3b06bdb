// libpqi core: set-up, weight preparation, gains, selection, single/double
// flip passes, flip application, fp64 re-scoring and bit packing (sm_100a).
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <climits>
#include <type_traits>

#include "pqi_common.cuh"
#include "pqi_tc.cuh"

namespace pqi {

static thread_local char g_last_error[256] = {0};

void set_error(cudaError_t e, const char* where) {
  snprintf(g_last_error, sizeof(g_last_error), "%s: %s", where, cudaGetErrorString(e));
}

void set_error_text(const char* msg) { snprintf(g_last_error, sizeof(g_last_error), "%s", msg); }

bool make_sel_geom(long count, int G, int L, SelGeom* out) {
  if (G <= 0 || L <= 0 || L > 64 || G % L != 0 || count < 0) return false;
  long long J = (count + G - 1) / G;
  if (J < 1) J = 1;
  if ((unsigned long long)G * (unsigned long long)J >= 0xFFFFFFFFull) return false;
  out->G = (uint32_t)G;
  out->L = (uint32_t)L;
  out->J = (uint32_t)J;
  memset(out->rank, 0xFF, sizeof(out->rank));
  memset(out->slot_of_rank, 0, sizeof(out->slot_of_rank));
  // Replay reduce_energy_index (kernels.cl:8-20) with every unranked slot tied:
  // slot t < off absorbs t + off only when t holds nothing better, i.e. a tie
  // keeps t. The slot that reaches 0 is the next in tie order.
  bool ranked[64] = {false};
  for (int r = 0; r < L; ++r) {
    bool present[64];
    int id[64];
    for (int t = 0; t < L; ++t) {
      present[t] = !ranked[t];
      id[t] = t;
    }
    for (int off = L >> 1; off > 0; off >>= 1) {
      for (int t = 0; t < off; ++t) {
        if (!present[t] && present[t + off]) {
          present[t] = true;
          id[t] = id[t + off];
        }
      }
    }
    if (!present[0]) break;
    out->rank[id[0]] = (uint8_t)r;
    out->slot_of_rank[r] = (uint8_t)id[0];
    ranked[id[0]] = true;
  }
  return true;
}

// ---------------------------------------------------------------------------
// Weight preparation

struct PrepStats {
  unsigned long long nonfinite;
  unsigned long long nonint;
  unsigned long long asym;
  unsigned int maxabs_bits;
  unsigned int pad;
};

// One 32x32 tile per block (32 x 8 threads): compares W[i][j] with W[j][i],
// classifies values and sums the upper triangle in float64.
__global__ void prep_scan_kernel(const float* __restrict__ W, int n, PrepStats* st,
                                 double* __restrict__ partial) {
  __shared__ float tT[32][33];
  __shared__ double red[256];
  __shared__ unsigned int red_u[3][256];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int bi = blockIdx.y, bj = blockIdx.x;
  // tile (bj, bi): rows bj*32.., cols bi*32..
  for (int r = ty; r < 32; r += 8) {
    const int row = bj * 32 + r, col = bi * 32 + tx;
    tT[r][tx] = (row < n && col < n) ? W[(size_t)row * n + col] : 0.0f;
  }
  __syncthreads();
  double up = 0.0;
  unsigned int nf = 0, ni = 0, as = 0;
  float mx = 0.0f;
  for (int r = ty; r < 32; r += 8) {
    const int i = bi * 32 + r, j = bj * 32 + tx;
    if (i < n && j < n) {
      const float w = W[(size_t)i * n + j];
      const float wt = tT[tx][r];  // W[j][i]
      if (!isfinite(w)) {
        ++nf;
      } else {
        if (i != j) {
          if (w != rintf(w)) ++ni;
          mx = fmaxf(mx, fabsf(w));
          if (w != wt) ++as;
          if (i < j) up += (double)w;
        }
      }
    }
  }
  const int tid = ty * 32 + tx;
  red[tid] = up;
  red_u[0][tid] = nf;
  red_u[1][tid] = ni;
  red_u[2][tid] = as;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (tid < s) {
      red[tid] += red[tid + s];
      red_u[0][tid] += red_u[0][tid + s];
      red_u[1][tid] += red_u[1][tid + s];
      red_u[2][tid] += red_u[2][tid + s];
    }
    __syncthreads();
  }
  if (tid == 0) {
    partial[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = red[0];
    if (red_u[0][0]) atomicAdd(&st->nonfinite, (unsigned long long)red_u[0][0]);
    if (red_u[1][0]) atomicAdd(&st->nonint, (unsigned long long)red_u[1][0]);
    if (red_u[2][0]) atomicAdd(&st->asym, (unsigned long long)red_u[2][0]);
  }
  // max |w|: non-negative floats order like their bit patterns
  unsigned int mb = __float_as_uint(mx);
  for (int o = 16; o > 0; o >>= 1) mb = max(mb, __shfl_xor_sync(0xFFFFFFFFu, mb, o));
  if (tx == 0 && mb) atomicMax(&st->maxabs_bits, mb);
}

// Deterministic sum of `count` doubles by one block.
__global__ void sum_partials_kernel(const double* __restrict__ p, size_t count, double* out) {
  __shared__ double red[1024];
  double s = 0.0;
  for (size_t i = threadIdx.x; i < count; i += blockDim.x) s += p[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x >> 1; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// Zero-diagonal, zero-padded copies with row pitch ld.
__global__ void prep_convert_kernel(const float* __restrict__ W, int n, int ld,
                                    float* __restrict__ Wz, int8_t* __restrict__ Wi8,
                                    uint16_t* __restrict__ Whi, uint16_t* __restrict__ Wlo) {
  const size_t total = (size_t)n * ld;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e / ld), j = (int)(e - (size_t)i * ld);
    const float w = (j < n && i != j) ? W[(size_t)i * n + j] : 0.0f;
    Wz[e] = w;
    if (Wi8) Wi8[e] = (int8_t)(int)w;
    if (Whi) {
      const __nv_bfloat16 hi = __float2bfloat16_rn(w);
      const __nv_bfloat16 lo = __float2bfloat16_rn(w - __bfloat162float(hi));
      Whi[e] = __bfloat16_as_ushort(hi);
      Wlo[e] = __bfloat16_as_ushort(lo);
    }
  }
}

// Fixed-point digit planes: v = rint(w * 2^S), |v| < 2^30, balanced int8
// digits v = d0 2^24 + d1 2^16 + d2 2^8 + d3 into four planes of n*ld bytes.
__global__ void prep_digits_kernel(const float* __restrict__ Wz, size_t total, double scale,
                                   int8_t* __restrict__ Wd) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    long long v = llrint((double)Wz[e] * scale);
#pragma unroll
    for (int p = 3; p > 0; --p) {
      const int d = (int)(((v + 128) & 255) - 128);
      Wd[(size_t)p * total + e] = (int8_t)d;
      v = (v - d) / 256;
    }
    Wd[e] = (int8_t)v;  // |v| <= 64 here
  }
}

// ---------------------------------------------------------------------------
// Gains: g_k = x_k * sum_v W_kv x_v, x = 2s - 1, one warp per row.

__device__ __forceinline__ double dot_bits(const float4& w, uint32_t bits4) {
  double a = 0.0;
  a += (bits4 & 1u) ? (double)w.x : -(double)w.x;
  a += (bits4 & 2u) ? (double)w.y : -(double)w.y;
  a += (bits4 & 4u) ? (double)w.z : -(double)w.z;
  a += (bits4 & 8u) ? (double)w.w : -(double)w.w;
  return a;
}

__device__ __forceinline__ int dot_bits_i8(const int4& w, uint32_t bits16) {
  int a = 0;
  const int32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int v = (int)(int8_t)((ws[q] >> (8 * b)) & 0xFF);
      a += ((bits16 >> (q * 4 + b)) & 1u) ? v : -v;
    }
  }
  return a;
}

// grid: (row blocks, count). Rows of the prepared copy have pitch ld.
template <typename WT>
__global__ void gains_gemv_kernel(const WT* __restrict__ Wp, int ld, int n,
                                  const uint32_t* __restrict__ theta, int n32,
                                  float* __restrict__ g32, double* __restrict__ g64) {
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  const uint32_t* th = theta + (size_t)blockIdx.y * n32;
  for (int k = blockIdx.x * warps + (threadIdx.x >> 5); k < n; k += gridDim.x * warps) {
    const WT* row = Wp + (size_t)k * ld;
    double acc = 0.0;
    if constexpr (sizeof(WT) == 4) {
      for (int v = lane * 4; v < n; v += 128) {
        const float4 w = *reinterpret_cast<const float4*>(row + v);
        const uint32_t b4 = (__ldg(th + (v >> 5)) >> (v & 31)) & 0xFu;
        acc += dot_bits(w, b4);
      }
    } else {
      int ai = 0;
      for (int v = lane * 16; v < n; v += 512) {
        const int4 w = *reinterpret_cast<const int4*>(row + v);
        const uint32_t b16 = (__ldg(th + (v >> 5)) >> (v & 31)) & 0xFFFFu;
        ai += dot_bits_i8(w, b16);
      }
      acc = (double)ai;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if (lane == 0) {
      const double g = get_bit32(th, k) ? acc : -acc;
      if (g32) g32[(size_t)blockIdx.y * n + k] = (float)g;
      if (g64) g64[(size_t)blockIdx.y * n + k] = g;
    }
  }
}

// ---------------------------------------------------------------------------
// Selection

__global__ void select_kernel(const float* __restrict__ vals, long long count, float scale,
                              SelGeom geo, unsigned long long* key) {
  __shared__ uint64_t scratch[32];
  uint64_t best = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    const uint64_t k = sel_key(vals[i] * scale, (uint64_t)i, geo);
    best = k > best ? k : best;
  }
  best = block_max_u64(best, scratch);
  if (threadIdx.x == 0 && best) atomicMax(key, (unsigned long long)best);
}

__global__ void select_finish_kernel(const unsigned long long* key, SelGeom geo, float* best_val,
                                     int* best_idx) {
  float v;
  int64_t i;
  sel_decode(*key, geo, &v, &i);
  if (best_val) *best_val = v;
  if (best_idx) *best_idx = (int)i;
}

// ---------------------------------------------------------------------------
// Double flips (kernels.cl:150-231 semantics, from maintained gains).
//
// Flipping k and l gains d = g_k + g_l - 2 x_k x_l W_kl; the reference's value
// is float(d) (x2 for a spin glass) and its selection is the maximum 64-bit
// key (sel_key) over all pairs k < l in k-major order.
//
// The upper triangle is cut into tiles of 16 rows x 1024 float32 columns
// (8 rows x 4096 int8 columns: 4 KB of each row), each W element read once.
// Every pair first gets an fp32 estimate a = f_k + f_l + c W_kl (f = the gain
// in the estimate's type, c = -2 when the bits agree, else +2). |a - value|
// is below 2^-22 (|g_k| + |g_l| + |a|), so a pair with a < thr - delta,
// delta = 2^-20 (max|g_k| + max|g_l| + |thr|), has value < thr; thr is a value
// some selectable pair (key != 0) reaches, so such a pair cannot be the
// maximum and is skipped. Only tiles holding a pair at the cut - the rare
// near-maxima - take pairs' exact float64 values and keys. thr is shared per
// block (shared memory) and across blocks (one global word), both as
// order-preserving uint32 under atomicMax, and seeded in every block from the
// pairs of the node with the largest gain.

constexpr int DS_ROWS = 16;  // rows per tile (float32 weights)

__device__ __forceinline__ float thr_of(uint32_t o) {
  // ordered 0 (nothing published yet) and anything below -inf read as -inf
  return o < ord_f32(-INFINITY) ? -INFINITY : unord_f32(o);
}

// Tie priority of pair index c under the reference geometry, from (t, j) =
// (c mod G, c / G); 32-bit (pair indices stay below 2^31 for n <= 46341).
__device__ __forceinline__ uint64_t pair_key(float v, uint32_t t, uint32_t j, const SelGeom& geo) {
  const uint32_t grp = t / geo.L;
  const uint32_t r = geo.rank[t - grp * geo.L];
  if (r == 0xFFu || v != v) return 0ull;
  return ((uint64_t)ord_f32(v) << 32) | (uint64_t)(0xFFFFFFFFu - ((grp * geo.L + r) * geo.J + j));
}

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may start once every CTA of the kernel before it has called
// launch_dependents; wait() then blocks until that kernel has completed and
// its writes are visible (a no-op without such a predecessor).
__device__ __forceinline__ void pdl_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Before the pass: the gains in the estimate's type (float32 for float
// weights, int32 - exact - for int8 weights), zero from n up to npad (the pass
// reads them as whole vectors), and per CTA two partials: the node of the
// largest gain (ordered gain << 32 | ~node, so the lowest node on ties) and the
// largest |gain| (ordered float32). CTA 0 also clears the pass's result key,
// shared threshold and CTA counter (ctl[0], ctl[1], ctl[3]): the pass touches
// them only after this kernel has completed.
template <typename WT>
__global__ void __launch_bounds__(256) double_prep_kernel(const double* __restrict__ g64, int n,
                                                          int npad, void* __restrict__ gest_v,
                                                          unsigned long long* __restrict__ parts,
                                                          unsigned long long* ctl) {
  constexpr bool INT = sizeof(WT) == 1;
  __shared__ uint64_t scratch[32];
  pdl_launch_dependents();  // the pass may start streaming W
  uint64_t am = 0, ga = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < npad; k += gridDim.x * blockDim.x) {
    if (k < n) {
      const double gk = g64[k];
      const float fk = (float)gk;
      if constexpr (INT) {
        static_cast<int*>(gest_v)[k] = (int)llrint(gk);
      } else {
        static_cast<float*>(gest_v)[k] = fk;
      }
      const uint64_t a = ((uint64_t)ord_f32(fk) << 32) | (uint64_t)(0xFFFFFFFFu - (uint32_t)k);
      am = a > am ? a : am;
      if (fk == fk) ga = max(ga, (uint64_t)ord_f32(fabsf(fk)));
    } else if constexpr (INT) {
      static_cast<int*>(gest_v)[k] = 0;
    } else {
      static_cast<float*>(gest_v)[k] = 0.0f;
    }
  }
  am = block_max_u64(am, scratch);
  ga = block_max_u64(ga, scratch);
  if (threadIdx.x == 0) {
    parts[blockIdx.x] = am;
    parts[gridDim.x + blockIdx.x] = ga;
    if (blockIdx.x == 0) {
      ctl[0] = 0ull;
      ctl[1] = 0ull;
      ctl[3] = 0ull;
    }
  }
}

// A first threshold close to the maximum: every pair (k, m) with the node m
// of the largest gain taken exactly - the best pairs usually contain the best
// single node, so few tiles then hold a pair at the cut. Every CTA folds the
// prep kernel's partials into m; W is symmetric, so W_km is read from row m.
// The pairs' keys go into the result, the largest selectable value into the
// shared threshold (one atomic per warp).
template <typename WT>
__global__ void __launch_bounds__(256) double_seed_kernel(
    const WT* __restrict__ Wp, int ld, int n, const uint32_t* __restrict__ theta,
    const double* __restrict__ g64, int spin, SelGeom geo,
    const unsigned long long* __restrict__ parts, int nparts, unsigned long long* key,
    unsigned int* gthr) {
  __shared__ uint64_t scratch[32];
  pdl_launch_dependents();  // the pass may start streaming W
  pdl_wait();               // the prep kernel's partials and cleared words
  uint64_t am = 0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    const uint64_t a = parts[i];
    am = a > am ? a : am;
  }
  am = block_max_u64(am, scratch);
  const int m = (int)(0xFFFFFFFFu - (uint32_t)am);
  const uint32_t xm = (uint32_t)get_bit32(theta, (uint32_t)m);
  const double gm = g64[m];
  const WT* __restrict__ rowm = Wp + (size_t)m * ld;
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int k = base + (int)threadIdx.x;
    uint64_t kk = 0;
    unsigned int o = 0;
    if (k < n && k != m) {
      const double wd = (double)rowm[k];
      const bool agree = (uint32_t)get_bit32(theta, (uint32_t)k) == xm;
      float v = (float)(g64[k] + gm - (agree ? 2.0 * wd : -2.0 * wd));
      const float vu = v;
      if (spin) v *= 2.0f;
      const int a = min(k, m), b = max(k, m);
      const uint32_t c = (uint32_t)(pair_base(a, n) + (long long)(b - a - 1));
      kk = pair_key(v, c % geo.G, c / geo.G, geo);
      if (kk != 0ull) o = ord_f32(vu);
    }
    kk = warp_max_u64(kk);
    o = __reduce_max_sync(0xFFFFFFFFu, o);
    if ((threadIdx.x & 31) == 0) {
      if (kk) atomicMax(key, (unsigned long long)kk);
      if (o) atomicMax(gthr, o);
    }
  }
}

// The pass streams W through shared memory: one persistent CTA per SM, a
// producer warp copying each tile's row segments of DS_ROW_BYTES
// (cp.async.bulk, completion counted on the stage's mbarrier) into a ring of
// DS_STAGES stages, and DS_CONSUMERS threads that score the tile from shared
// memory (the estimate, then the exact path for the rare flagged rows) and
// release the stage. The copies run up to DS_STAGES tiles ahead of the
// scoring, so HBM sees a deep queue of large requests whatever the scoring's
// latency.
constexpr int DS_STAGES = 3;
constexpr int DS_CONSUMERS = 256;
constexpr int DS_THREADS = DS_CONSUMERS + 32;
constexpr int DS_ROW_BYTES = 16 * DS_CONSUMERS;  // 4 KB of a row per tile
constexpr int DS_TILE_BYTES = DS_ROWS * DS_ROW_BYTES;
constexpr int DS_SMEM = DS_STAGES * DS_TILE_BYTES;
constexpr int DS_CTAS_PER_SM = 1;  // resident pass CTAs per SM
// the gains in the estimate's type are padded to a multiple of this many
// entries (a whole tile's columns for either weight type)
constexpr int DS_GEST_PAD = 4096;

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          tc::smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(tc::smem_u32(bar))
      : "memory");
}

// Packed float32 pairs: d = a * b + c per half, round to nearest (the same
// rounding as fmaf on each half).
__device__ __forceinline__ uint64_t pack2(float lo, float hi) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void unpack2(uint64_t v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}

// The pass's tiles: the kept tiles (those reaching above the diagonal,
// (c + 1) CW > rg DR + 1, i.e. chunks c >= rg / (CW / DR) of row group rg) in
// row group major order, cut into gridDim.x contiguous runs, one per CTA.
// Each CTA so streams its own rows chunk after chunk, and at any time the
// CTAs read rows spread over the whole triangle (measured faster than
// interleaving the CTAs tile by tile). The start of a run is found by a
// binary search on the closed-form count of kept tiles before a row group.
// The producer and the consumers walk the same run.
template <int CW, int DR>
struct TileWalk {
  int ng, nc, rg, c, left;
  // kept tiles of row groups 0 .. R-1 (row group r keeps chunks r / Q .. nc-1)
  __device__ __forceinline__ long long prefix(long long R) const {
    constexpr long long Q = CW / DR;
    const long long a = R / Q, r = R - (R / Q) * Q;
    return R * nc - (Q * a * (a - 1) / 2 + a * r);
  }
  __device__ __forceinline__ TileWalk(int n, int b, int G) {
    ng = (n - 1 + DR - 1) / DR;
    nc = (n + CW - 1) / CW;
    const long long total = prefix(ng);
    const long long T = (total + G - 1) / G;
    const long long t0 = (long long)b * T;
    const long long t1 = t0 + T < total ? t0 + T : total;
    left = t1 > t0 ? (int)(t1 - t0) : 0;
    rg = ng;
    c = 0;
    if (!left) return;
    int lo = 0, hi = ng - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (prefix(mid) <= t0) {
        lo = mid;
      } else {
        hi = mid - 1;
      }
    }
    rg = lo;
    c = rg / (CW / DR) + (int)(t0 - prefix(rg));
  }
  __device__ __forceinline__ bool valid() const { return left > 0; }
  __device__ __forceinline__ void next() {
    --left;
    if (++c == nc) {
      ++rg;
      c = rg / (CW / DR);
    }
  }
};

template <typename WT>
__global__ void __launch_bounds__(DS_THREADS, DS_CTAS_PER_SM) double_stream_kernel(
    const WT* __restrict__ Wp, int ld, int n, const uint32_t* __restrict__ theta,
    const double* __restrict__ g64, const void* __restrict__ gest_v,
    const unsigned long long* __restrict__ parts, int nparts, int spin, SelGeom geo,
    unsigned long long* key, unsigned int* gthr, unsigned int* done, float* best_val,
    int* best_idx) {
  constexpr int VEC = 16 / (int)sizeof(WT);  // columns per consumer thread
  constexpr int CW = VEC * DS_CONSUMERS;    // columns per tile (DS_ROW_BYTES of a row)
  constexpr bool INT = sizeof(WT) == 1;
  // rows per tile: 16 for float32 (64 KB stages), 8 for int8 (its graphs are
  // small and L2-resident: more, smaller tiles keep every SM busy)
  constexpr int DR = INT ? 8 : DS_ROWS;
  typedef typename std::conditional<INT, int, float>::type ET;
  const ET* __restrict__ gest = static_cast<const ET*>(gest_v);
  extern __shared__ __align__(1024) unsigned char ring[];
  __shared__ __align__(8) uint64_t full_bar[DS_STAGES];
  __shared__ __align__(8) uint64_t empty_bar[DS_STAGES];
  __shared__ uint64_t scratch[32];
  __shared__ unsigned int s_thr;
  __shared__ int s_fail;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int st = 0; st < DS_STAGES; ++st) {
      tc::mbar_init(&full_bar[st], 1);
      tc::mbar_init(&empty_bar[st], DS_CONSUMERS / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    s_thr = 0u;
    s_fail = 0;
  }
  __syncthreads();
  uint64_t best = 0;
  if (warp == DS_CONSUMERS / 32) {
    // producer: this CTA's tiles, each into the next stage once the
    // consumers released it. W is not written by the kernels before this
    // one, so the copies start at once
    if (lane == 0) {
      int it = 0;
      for (TileWalk<CW, DR> tw(n, blockIdx.x, gridDim.x); tw.valid(); tw.next()) {
        const int rg = tw.rg, c = tw.c;
        const int st = it % DS_STAGES;
        const uint32_t use = (uint32_t)(it / DS_STAGES);
        if (use > 0 && !tc::mbar_wait(&empty_bar[st], (use - 1) & 1u)) {
          s_fail = 1;
          break;
        }
        // the row segments from the first column above the tile's first row
        // (rounded down to 16 bytes) to the chunk's end, within the padded
        // row (ld is a multiple of 128); column l sits at (l - col0) of its
        // row's slot either way
        const int col0 = c * CW;
        const int cs = max(col0, (rg * DR + 1) & ~(16 / (int)sizeof(WT) - 1));
        const uint32_t bytes = (uint32_t)((min(col0 + CW, ld) - cs) * (int)sizeof(WT));
        tc::mbar_expect_tx(&full_bar[st], bytes * DR);
        unsigned char* dst = ring + (size_t)st * DS_TILE_BYTES + (size_t)(cs - col0) * sizeof(WT);
#pragma unroll
        for (int i = 0; i < DR; ++i) {
          const int k = min(rg * DR + i, n - 1);
          bulk_copy_g2s(dst + i * DS_ROW_BYTES, Wp + (size_t)k * ld + cs, bytes, &full_bar[st]);
        }
        ++it;
      }
    }
  } else {
    // consumers: wait for the kernels before this one (the gains in the
    // estimate's type, the prep kernel's partials, the seeded threshold);
    // the producer does not
    pdl_wait();
    // the largest |gain| (every warp folds the prep kernel's partials itself)
    uint64_t ga = 0;
    for (int i = lane; i < nparts; i += 32) {
      const uint64_t b = parts[nparts + i];
      ga = b > ga ? b : ga;
    }
    ga = warp_max_u64(ga);
    const float gabs = ga ? unord_f32((uint32_t)ga) : 0.0f;
    float thr = thr_of(__ldcg(gthr));
    // Each tile's row gains and bits, this thread's column gains and bits and
    // the shared threshold are loaded one tile ahead, so their latency hides
    // behind the tile before (the gains are padded: rows and columns past n
    // read zeros)
    ET fk[DR], fl[VEC];
    uint32_t xk = 0, lw = 0;
    unsigned int gt = 0;
    TileWalk<CW, DR> tw(n, blockIdx.x, gridDim.x);
    auto load_header = [&](int rg_, int c_) {
      const int k0_ = rg_ * DR;
#pragma unroll
      for (int q = 0; q < DR / 4; ++q) {
        const int4 v = __ldg(reinterpret_cast<const int4*>(gest + k0_) + q);
        memcpy(&fk[4 * q], &v, 16);
      }
      xk = __ldg(theta + (k0_ >> 5)) >> (k0_ & 31);
      const int l0_ = c_ * CW + (int)threadIdx.x * VEC;
#pragma unroll
      for (int q = 0; q < VEC / 4; ++q) {
        const int4 v = __ldg(reinterpret_cast<const int4*>(gest + l0_) + q);
        memcpy(&fl[4 * q], &v, 16);
      }
      lw = l0_ < n ? __ldg(theta + (l0_ >> 5)) >> (l0_ & 31) : 0u;
      gt = __ldcg(gthr);
    };
    if (tw.valid()) load_header(tw.rg, tw.c);
    int it = 0;
    while (tw.valid()) {
      const int rg = tw.rg, c = tw.c;
      const int st = it % DS_STAGES;
      const uint32_t use = (uint32_t)(it / DS_STAGES);
      ++it;
      const int k0 = rg * DR;
      const int l0 = c * CW + (int)threadIdx.x * VEC;
      ET fkc[DR], flc[VEC];
#pragma unroll
      for (int i = 0; i < DR; ++i) fkc[i] = fk[i];
#pragma unroll
      for (int e = 0; e < VEC; ++e) flc[e] = fl[e];
      const uint32_t xkc = xk, lwc = lw;
      thr = fmaxf(thr, thr_of(max(*(volatile unsigned int*)&s_thr, gt)));
      tw.next();
      if (tw.valid()) load_header(tw.rg, tw.c);
      if (!tc::mbar_wait_warp(&full_bar[st], use & 1u)) {
        s_fail = 1;
        break;
      }
      const unsigned char* tile = ring + (size_t)st * DS_TILE_BYTES + threadIdx.x * 16;
      WT w[DR][VEC];
#pragma unroll
      for (int i = 0; i < DR; ++i) {
        const int4 v = *reinterpret_cast<const int4*>(tile + i * DS_ROW_BYTES);
        memcpy(&w[i][0], &v, 16);
      }
      // |estimate - value| <= 2^-22 (|g_k| + |g_l| + |value|) <= 2^-22 (2 max|g| + |value|)
      float cut = INT ? thr : thr - (2.0f * gabs + fabsf(thr)) * 9.5367431640625e-07f;
      int cut_i = thr > -INFINITY ? (int)thr : INT_MIN;
      // each row's largest estimate f_k + max_l (f_l -/+ 2 W_kl) over this
      // thread's columns. The coefficient of W_kl is -2 where the bits agree,
      // else +2: for a row with bit 1 that is cp[e] (from column l's bit),
      // for a row with bit 0 its negation. The rows' bits are the same for
      // every thread, so the branch on them is uniform. (The grouping differs
      // from the exact path's (f_k + f_l) -/+ 2 W by a few units in the last
      // place, far inside the cut's 2^-20 margin.)
      ET ra[DR];
      bool any;
      if constexpr (INT) {
        int cp[VEC];
#pragma unroll
        for (int e = 0; e < VEC; ++e) cp[e] = ((lwc >> e) & 1u) ? -2 : 2;
        int amax = INT_MIN;
#pragma unroll
        for (int i = 0; i < DR; ++i) {
          int r;
          if ((xkc >> i) & 1u) {
            r = flc[0] + cp[0] * (int)w[i][0];
#pragma unroll
            for (int e = 1; e < VEC; ++e) r = max(r, flc[e] + cp[e] * (int)w[i][e]);
          } else {
            r = flc[0] - cp[0] * (int)w[i][0];
#pragma unroll
            for (int e = 1; e < VEC; ++e) r = max(r, flc[e] - cp[e] * (int)w[i][e]);
          }
          ra[i] = fkc[i] + r;
          amax = max(amax, ra[i]);
        }
        any = amax >= cut_i;
      } else {
        // two columns per packed f32x2 FMA
        const float c0 = ((lwc >> 0) & 1u) ? -2.0f : 2.0f, c1 = ((lwc >> 1) & 1u) ? -2.0f : 2.0f;
        const float c2 = ((lwc >> 2) & 1u) ? -2.0f : 2.0f, c3 = ((lwc >> 3) & 1u) ? -2.0f : 2.0f;
        const uint64_t cp01 = pack2(c0, c1), cp23 = pack2(c2, c3);
        const uint64_t cn01 = pack2(-c0, -c1), cn23 = pack2(-c2, -c3);
        const uint64_t fl01 = pack2(flc[0], flc[1]), fl23 = pack2(flc[2], flc[3]);
#pragma unroll
        for (int i = 0; i < DR; ++i) {
          const uint64_t w01 = pack2(w[i][0], w[i][1]), w23 = pack2(w[i][2], w[i][3]);
          uint64_t d01, d23;
          if ((xkc >> i) & 1u) {
            d01 = fma2(cp01, w01, fl01);
            d23 = fma2(cp23, w23, fl23);
          } else {
            d01 = fma2(cn01, w01, fl01);
            d23 = fma2(cn23, w23, fl23);
          }
          float d0, d1, d2, d3;
          unpack2(d01, d0, d1);
          unpack2(d23, d2, d3);
          ra[i] = fkc[i] + max3f(d0, d1, fmaxf(d2, d3));
        }
        float amax = max3f(ra[0], ra[1], ra[2]);
#pragma unroll
        for (int i = 3; i + 1 < DR; i += 2) amax = max3f(amax, ra[i], ra[i + 1]);
        if constexpr (DR % 2 == 0) amax = fmaxf(amax, ra[DR - 1]);
        any = amax >= cut;
      }
      // (columns before the copied part hold stale bytes: every pair there
      // has l <= k, and a thread with no column after the copy start has
      // none; columns past the copied row segment likewise: such a thread
      // has no column below n)
      if (any && l0 < n && l0 + VEC > max(c * CW, (k0 + 1) & ~(VEC - 1))) {
        const WT* tw_ = reinterpret_cast<const WT*>(ring + (size_t)st * DS_TILE_BYTES);
        // only the rows whose largest estimate reaches the cut
        uint32_t rows = 0u;
#pragma unroll
        for (int i = 0; i < DR; ++i) {
          if constexpr (INT) {
            rows |= (uint32_t)(ra[i] >= cut_i) << i;
          } else {
            rows |= (uint32_t)(ra[i] >= cut) << i;
          }
        }
#pragma unroll 1
        for (int b = 0; b < DR * VEC; ++b) {
          const int i = b / VEC, e = b % VEC;
          if (!((rows >> i) & 1u)) {
            b += VEC - 1 - e;  // the rest of the row
            continue;
          }
          const int k = k0 + i, l = l0 + e;
          if (k >= n - 1 || l <= k || l >= n) continue;
          const WT wv = tw_[i * (DS_ROW_BYTES / (int)sizeof(WT)) + (l - c * CW)];
          const uint32_t flip = (((xkc >> i) & 1u) ^ ((lwc >> e) & 1u)) ^ 1u;
          float v;
          if constexpr (INT) {
            const int ai = __ldg(gest + k) + __ldg(gest + l) + (flip ? -2 * (int)wv : 2 * (int)wv);
            if (ai < cut_i) continue;
            v = (float)ai;
          } else {
            const float cw = __uint_as_float(__float_as_uint(wv) ^ (flip << 31));
            if (fmaf(2.0f, cw, __ldg(gest + k) + __ldg(gest + l)) < cut) continue;
            const double wd = (double)wv;
            v = (float)(__ldg(g64 + k) + __ldg(g64 + l) - (flip ? 2.0 * wd : -2.0 * wd));
          }
          const float vu = v;
          if (spin) v *= 2.0f;
          const uint32_t cidx = (uint32_t)(pair_base(k, n) + (long long)(l - k - 1));
          const uint64_t kk = pair_key(v, cidx % geo.G, cidx / geo.G, geo);
          best = kk > best ? kk : best;
          if (kk != 0ull && vu > thr) {
            thr = vu;
            cut = INT ? thr : thr - (2.0f * gabs + fabsf(thr)) * 9.5367431640625e-07f;
            cut_i = (int)thr;
          }
        }
      }
      // the stage back to the producer (this warp's reads are done)
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&empty_bar[st]);
      if (thr > -INFINITY) {
        const unsigned int o = ord_f32(thr);
        if (o > *(volatile unsigned int*)&s_thr) {
          atomicMax(&s_thr, o);
          if (o > __ldcg(gthr)) atomicMax(gthr, o);
        }
      }
    }
  }
  best = block_max_u64(best, scratch);
  // a wait that ran out leaves no result (key 0: value -inf, index -1); the
  // last CTA to finish decodes the selection
  if (threadIdx.x == 0) {
    if (best && !s_fail) atomicMax(key, (unsigned long long)best);
    __threadfence();
    if (atomicAdd(done, 1u) == gridDim.x - 1) {
      __threadfence();
      float v;
      int64_t i;
      sel_decode(*(volatile unsigned long long*)key, geo, &v, &i);
      if (best_val) *best_val = v;
      if (best_idx) *best_idx = (int)i;
    }
  }
}

// Apply one or two flips to (theta, gains64). x = 2s - 1 of the state before.
template <typename WT>
__global__ void apply_flip_gains_kernel(const WT* __restrict__ Wp, int ld, int n,
                                        const uint32_t* __restrict__ theta,
                                        double* __restrict__ g64, int k, int l) {
  const double xk = get_bit32(theta, k) ? 1.0 : -1.0;
  const double xl = (l >= 0) ? (get_bit32(theta, l) ? 1.0 : -1.0) : 0.0;
  const WT* rk = Wp + (size_t)k * ld;
  const WT* rl = (l >= 0) ? Wp + (size_t)l * ld : nullptr;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const double xv = get_bit32(theta, v) ? 1.0 : -1.0;
    double g = g64[v];
    if (l < 0) {
      g = (v == k) ? -g : g - 2.0 * xv * xk * (double)rk[v];
    } else if (v == k) {
      g = -g + 2.0 * xk * xl * (double)rl[k];
    } else if (v == l) {
      g = -(g - 2.0 * xl * xk * (double)rk[l]);
    } else {
      g = g - 2.0 * xv * xk * (double)rk[v] - 2.0 * xv * xl * (double)rl[v];
    }
    g64[v] = g;
  }
}

__global__ void toggle_bits_kernel(uint32_t* theta, int k, int l) {
  theta[k >> 5] ^= 1u << (k & 31);
  if (l >= 0) theta[l >> 5] ^= 1u << (l & 31);
}

// ---------------------------------------------------------------------------
// fp64 re-scoring against the caller's W (diagonal included).
// grid (row blocks, count); warp per row; partial[b][blk] = (D, T).

__global__ void rescore_kernel(const float* __restrict__ W, int n,
                               const uint32_t* __restrict__ theta, int n32,
                               double* __restrict__ partial) {
  __shared__ double sd[32], stt[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int warps = blockDim.x >> 5;
  const uint32_t* th = theta + (size_t)blockIdx.y * n32;
  double d = 0.0, t = 0.0;
  for (int u = blockIdx.x * warps + warp; u < n; u += gridDim.x * warps) {
    const float* row = W + (size_t)u * n;
    const int su = get_bit32(th, u);
    for (int v = lane; v < n; v += 32) {
      const double w = (double)row[v];
      t += w;
      if (get_bit32(th, v) != su) d += w;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    d += __shfl_xor_sync(0xFFFFFFFFu, d, o);
    t += __shfl_xor_sync(0xFFFFFFFFu, t, o);
  }
  if (lane == 0) {
    sd[warp] = d;
    stt[warp] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double D = 0.0, T = 0.0;
    for (int w = 0; w < warps; ++w) {
      D += sd[w];
      T += stt[w];
    }
    double* p = partial + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 2;
    p[0] = D;
    p[1] = T;
  }
}

__global__ void rescore_finish_kernel(const double* __restrict__ partial, int nblk, int count,
                                      double* cut, double* energy) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= count) return;
  double D = 0.0, T = 0.0;
  for (int i = 0; i < nblk; ++i) {
    D += partial[((size_t)b * nblk + i) * 2];
    T += partial[((size_t)b * nblk + i) * 2 + 1];
  }
  if (cut) cut[b] = D / 2.0;
  if (energy) energy[b] = D - T / 2.0;
}

// ---------------------------------------------------------------------------
// Packing

__global__ void pack_kernel(const uint8_t* __restrict__ bools, int rows, int n, int n32,
                            uint32_t* __restrict__ words) {
  const long long total = (long long)rows * n32;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e / n32), w = (int)(e - (long long)r * n32);
    const uint8_t* src = bools + (size_t)r * n + (size_t)w * 32;
    const int lim = min(32, n - w * 32);
    uint32_t acc = 0;
    for (int b = 0; b < lim; ++b) acc |= (src[b] ? 1u : 0u) << b;
    words[e] = acc;
  }
}

__global__ void unpack_kernel(const uint32_t* __restrict__ words, int rows, int n, int n32,
                              uint8_t* __restrict__ bools) {
  const long long total = (long long)rows * n;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e / n), j = (int)(e - (long long)r * n);
    bools[e] = (words[(size_t)r * n32 + (j >> 5)] >> (j & 31)) & 1u;
  }
}

static int grid_for(long long work, int block, int cap = 148 * 16) {
  long long g = (work + block - 1) / block;
  if (g < 1) g = 1;
  return (int)std::min<long long>(g, cap);
}

// Host helpers shared with the other translation units.
pqi_status launch_gains(const pqi_weights* w, const uint32_t* theta, int count, float* g32,
                        double* g64, cudaStream_t s) {
  const int n = w->n, n32 = (n + 31) >> 5;
  dim3 block(256);
  dim3 grid((unsigned)std::max(1, std::min((n + 7) / 8, 148 * 4)), (unsigned)count);
  if (w->kind == PQI_W_I8) {
    gains_gemv_kernel<int8_t><<<grid, block, 0, s>>>(w->W_i8, w->ld, n, theta, n32, g32, g64);
  } else {
    gains_gemv_kernel<float><<<grid, block, 0, s>>>(w->W_f32z, w->ld, n, theta, n32, g32, g64);
  }
  PQI_LAUNCHED("gains_gemv_kernel");
  return PQI_OK;
}

pqi_status launch_select(const float* vals, long long count, float scale, const SelGeom& geo,
                         unsigned long long* key, float* best_val, int* best_idx,
                         cudaStream_t s) {
  PQI_TRY(cudaMemsetAsync(key, 0, sizeof(unsigned long long), s));
  select_kernel<<<grid_for(count, 256, 148 * 8), 256, 0, s>>>(vals, count, scale, geo, key);
  PQI_LAUNCHED("select_kernel");
  select_finish_kernel<<<1, 1, 0, s>>>(key, geo, best_val, best_idx);
  PQI_LAUNCHED("select_finish_kernel");
  return PQI_OK;
}

}  // namespace pqi

using namespace pqi;

extern "C" {

const char* pqi_version(void) { return "libpqi 0.1 (sm_100a)"; }

const char* pqi_last_error(void) { return g_last_error; }

pqi_status pqi_check_device(int device) {
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return PQI_ECUDA;
  if (p.major != 10) return PQI_ENOTSUP;
  return PQI_OK;
}

int pqi_padded_ld(int n) { return ((n + 127) / 128) * 128; }

size_t pqi_workspace_bytes(int n, long count) {
  if (n < 1) n = 1;
  if (count < 1) count = 1;
  const size_t ld = (size_t)pqi_padded_ld(n);
  const size_t cnt_pad = ((size_t)count + 127) / 128 * 128;
  size_t b = 1 << 16;                                   // scalars, keys, stats
  b += cnt_pad * ld * 4;                                // expanded +-1 operand (bf16 x2 worst case)
  b += ((size_t)ld / 64 + 2) * (size_t)count * 8;       // per-tile partial scores
  b += (size_t)count * 4 + 256;                         // per-candidate energies
  b += (size_t)n * 8 * 2 + 512;                         // base gains (f64) and f32 copy
  const size_t tiles = (size_t)((n + 31) / 32) * ((n + 31) / 32);
  const size_t nblk = (size_t)std::max(1, std::min((n + 7) / 8, 2048));
  size_t extra = std::max(tiles * 8, (size_t)count * nblk * 16);  // prep / rescore partials
  if (n > 24576) extra = std::max(extra, (size_t)count * n * 8);  // gray gains in global memory
  b += extra;
  return b;
}

pqi_status pqi_scan_weights(const float* W, int n, void* workspace, size_t workspace_bytes,
                            pqi_weight_stats* out, void* stream) {
  PQI_CHECK_ARG(W && out && n > 0);
  cudaStream_t s = as_stream(stream);
  Workspace ws(workspace, workspace_bytes);
  PrepStats* st = ws.take<PrepStats>(1);
  double* sum = ws.take<double>(1);
  const int tb = (n + 31) / 32;
  double* partial = ws.take<double>((size_t)tb * tb);
  PQI_CHECK_ARG(st && sum && partial);
  PQI_TRY(cudaMemsetAsync(st, 0, sizeof(PrepStats), s));
  prep_scan_kernel<<<dim3(tb, tb), dim3(32, 8), 0, s>>>(W, n, st, partial);
  PQI_LAUNCHED("prep_scan_kernel");
  sum_partials_kernel<<<1, 1024, 0, s>>>(partial, (size_t)tb * tb, sum);
  PQI_LAUNCHED("sum_partials_kernel");
  PrepStats hs;
  double hsum = 0.0;
  PQI_TRY(cudaMemcpyAsync(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost, s));
  PQI_TRY(cudaMemcpyAsync(&hsum, sum, sizeof(hsum), cudaMemcpyDeviceToHost, s));
  PQI_TRY(cudaStreamSynchronize(s));
  out->nonfinite = hs.nonfinite;
  out->nonint = hs.nonint;
  out->asym = hs.asym;
  memcpy(&out->maxabs, &hs.maxabs_bits, 4);
  out->kind = (hs.nonint == 0 && out->maxabs <= 127.0f) ? PQI_W_I8 : PQI_W_F32;
  out->upper_sum = hsum;
  if (hs.nonfinite || hs.asym) return PQI_EINVAL;
  return PQI_OK;
}

pqi_status pqi_prepare_weights(const float* W, int n, const pqi_weight_stats* stats,
                               float* W_f32z, int8_t* W_i8, uint16_t* W_hi, uint16_t* W_lo,
                               pqi_weights* out, void* stream) {
  PQI_CHECK_ARG(W && W_f32z && out && stats && n > 0);
  PQI_CHECK_ARG(stats->nonfinite == 0 && stats->asym == 0);
  const bool as_int8 = stats->kind == PQI_W_I8;
  if (as_int8) {
    PQI_CHECK_ARG(W_i8);
  } else {
    PQI_CHECK_ARG(W_hi && W_lo);
  }
  cudaStream_t s = as_stream(stream);
  const int ld = pqi_padded_ld(n);
  prep_convert_kernel<<<grid_for((long long)n * ld, 256, 148 * 16), 256, 0, s>>>(
      W, n, ld, W_f32z, as_int8 ? W_i8 : nullptr, as_int8 ? nullptr : W_hi,
      as_int8 ? nullptr : W_lo);
  PQI_LAUNCHED("prep_convert_kernel");
  out->W = W;
  out->W_f32z = W_f32z;
  out->W_i8 = as_int8 ? W_i8 : nullptr;
  out->W_hi = as_int8 ? nullptr : W_hi;
  out->W_lo = as_int8 ? nullptr : W_lo;
  out->n = n;
  out->ld = ld;
  out->kind = as_int8 ? PQI_W_I8 : PQI_W_F32;
  out->upper_sum = stats->upper_sum;
  out->W_d = nullptr;  // pqi_prepare_digits fills these
  out->wscale = 1.0;
  return PQI_OK;
}

pqi_status pqi_prepare_digits(pqi_weights* w, float maxabs, int8_t* W_d, void* stream) {
  PQI_CHECK_ARG(w && W_d && w->W_f32z && w->kind == PQI_W_F32 && w->n > 0 && maxabs >= 0.0f &&
                std::isfinite(maxabs));
  // largest S with maxabs * 2^S < 2^30 - 1 (rounding then stays below 2^30)
  const double lim = 1073741823.0;
  int S = 0;
  if (maxabs > 0.0f) {
    int e = 0;
    std::frexp((double)maxabs, &e);  // maxabs = f 2^e, f in [0.5, 1)
    S = 29 - e;                       // maxabs 2^S < 2^29
    while (std::ldexp((double)maxabs, S + 1) < lim) ++S;
    while (std::ldexp((double)maxabs, S) >= lim) --S;
  }
  const size_t total = (size_t)w->n * w->ld;
  prep_digits_kernel<<<grid_for((long long)total, 256, 148 * 16), 256, 0, as_stream(stream)>>>(
      w->W_f32z, total, std::ldexp(1.0, S), W_d);
  PQI_LAUNCHED("prep_digits_kernel");
  w->W_d = W_d;
  w->wscale = std::ldexp(1.0, -S);
  return PQI_OK;
}

pqi_status pqi_gains(const pqi_weights* w, const uint32_t* theta, int count, float* gains,
                     double* gains64, void* workspace, size_t workspace_bytes, void* stream) {
  (void)workspace;
  (void)workspace_bytes;
  PQI_CHECK_ARG(w && theta && count > 0 && (gains || gains64));
  return launch_gains(w, theta, count, gains, gains64, as_stream(stream));
}

pqi_status pqi_select(const float* values, long count, int global_size, int local_size,
                      float* best_value, int* best_index, void* workspace,
                      size_t workspace_bytes, void* stream) {
  PQI_CHECK_ARG(values && count > 0);
  SelGeom geo;
  PQI_CHECK_ARG(make_sel_geom(count, global_size, local_size, &geo));
  Workspace ws(workspace, workspace_bytes);
  unsigned long long* key = ws.take<unsigned long long>(1);
  PQI_CHECK_ARG(key);
  return launch_select(values, count, 1.0f, geo, key, best_value, best_index, as_stream(stream));
}

pqi_status pqi_select_host(const float* values_host, long count, int global_size, int local_size,
                           float* best_value_host, int* best_index_host) {
  PQI_CHECK_ARG(values_host && count > 0 && best_value_host && best_index_host);
  SelGeom geo;
  PQI_CHECK_ARG(make_sel_geom(count, global_size, local_size, &geo));
  uint64_t best = 0;
  for (long i = 0; i < count; ++i) {
    const uint64_t k = sel_key(values_host[i], (uint64_t)i, geo);
    best = k > best ? k : best;
  }
  float v;
  int64_t idx;
  sel_decode(best, geo, &v, &idx);
  *best_value_host = v;
  *best_index_host = (int)idx;
  return PQI_OK;
}

pqi_status pqi_single_bit_flips(const pqi_weights* w, const uint32_t* theta, int is_spin_glass,
                                int global_size, int local_size, float* best_energy,
                                int* best_index, void* workspace, size_t workspace_bytes,
                                void* stream) {
  PQI_CHECK_ARG(w && theta);
  SelGeom geo;
  PQI_CHECK_ARG(make_sel_geom(w->n, global_size, local_size, &geo));
  Workspace ws(workspace, workspace_bytes);
  unsigned long long* key = ws.take<unsigned long long>(1);
  float* g32 = ws.take<float>(w->n);
  PQI_CHECK_ARG(key && g32);
  cudaStream_t s = as_stream(stream);
  pqi_status rc = launch_gains(w, theta, 1, g32, nullptr, s);
  if (rc) return rc;
  return launch_select(g32, w->n, is_spin_glass ? 2.0f : 1.0f, geo, key, best_energy, best_index,
                       s);
}

pqi_status pqi_double_bit_flips(const pqi_weights* w, const uint32_t* theta,
                                const double* gains64, int is_spin_glass, int global_size,
                                int local_size, float* best_energy, int* best_index,
                                void* workspace, size_t workspace_bytes, void* stream) {
  PQI_CHECK_ARG(w && theta && w->n >= 2 && w->n <= 46341);
  const int n = w->n;
  const long long combo = (long long)n * (n - 1) / 2;
  SelGeom geo;
  PQI_CHECK_ARG(make_sel_geom(combo, global_size, local_size, &geo));
  Workspace ws(workspace, workspace_bytes);
  // the result key, the threshold word, a spare word, the CTA counter
  unsigned long long* key = ws.take<unsigned long long>(4);
  PQI_CHECK_ARG(key);
  cudaStream_t s = as_stream(stream);
  if (!gains64) {
    double* g = ws.take<double>(n);
    PQI_CHECK_ARG(g);
    pqi_status rc = launch_gains(w, theta, 1, nullptr, g, s);
    if (rc) return rc;
    gains64 = g;
  }
  // the gains in the estimate's type (4 bytes each), padded for whole-vector
  // reads, and the prep kernel's per-CTA partials
  const int npad = (n + DS_GEST_PAD - 1) / DS_GEST_PAD * DS_GEST_PAD;
  void* gest = ws.take<float>(npad);
  PQI_CHECK_ARG(gest);
  const int pg = grid_for(npad, 256, 148);
  unsigned long long* parts = ws.take<unsigned long long>(2 * (size_t)pg);
  PQI_CHECK_ARG(parts);
  // the result key, the shared threshold (key[1]) and the CTA counter
  // (key[3]) are cleared by the prep kernel; the seed kernel and the pass
  // are launched as programmatic dependents: the pass's producer streams W
  // while the gains are converted and the threshold seeded, its consumers
  // wait for both (pdl_wait)
  unsigned int* gthr = reinterpret_cast<unsigned int*>(key + 1);
  unsigned int* done = reinterpret_cast<unsigned int*>(key + 3);
  const int i8 = w->kind == PQI_W_I8 ? 1 : 0;
  cudaLaunchAttribute pdl[1];
  pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  pdl[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t seed_cfg = {};
  seed_cfg.gridDim = dim3(grid_for(n, 256, 148 * 4));
  seed_cfg.blockDim = dim3(256);
  seed_cfg.stream = s;
  seed_cfg.attrs = pdl;
  seed_cfg.numAttrs = 1;
  if (i8) {
    double_prep_kernel<int8_t><<<pg, 256, 0, s>>>(gains64, n, npad, gest, parts, key);
    PQI_LAUNCHED("double_prep_kernel");
    PQI_TRY(cudaLaunchKernelEx(&seed_cfg, double_seed_kernel<int8_t>, (const int8_t*)w->W_i8, w->ld,
                               n, theta, gains64, is_spin_glass, geo,
                               (const unsigned long long*)parts, pg, key, gthr));
  } else {
    double_prep_kernel<float><<<pg, 256, 0, s>>>(gains64, n, npad, gest, parts, key);
    PQI_LAUNCHED("double_prep_kernel");
    PQI_TRY(cudaLaunchKernelEx(&seed_cfg, double_seed_kernel<float>, (const float*)w->W_f32z, w->ld,
                               n, theta, gains64, is_spin_glass, geo,
                               (const unsigned long long*)parts, pg, key, gthr));
  }
  PQI_LAUNCHED("double_seed_kernel");
  // persistent CTAs, DS_CTAS_PER_SM per SM (the stage rings take most of
  // shared memory)
  static int sms = 0;
  static bool attr_set[2] = {false, false};
  if (!sms) {
    int dev = 0;
    PQI_TRY(cudaGetDevice(&dev));
    PQI_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  }
  if (!attr_set[i8]) {
    const void* fn = i8 ? (const void*)double_stream_kernel<int8_t> : (const void*)double_stream_kernel<float>;
    PQI_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, DS_SMEM));
    attr_set[i8] = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(sms * DS_CTAS_PER_SM);
  cfg.blockDim = dim3(DS_THREADS);
  cfg.dynamicSmemBytes = DS_SMEM;
  cfg.stream = s;
  cfg.attrs = pdl;
  cfg.numAttrs = 1;
  if (i8) {
    PQI_TRY(cudaLaunchKernelEx(&cfg, double_stream_kernel<int8_t>, (const int8_t*)w->W_i8, w->ld, n,
                               theta, gains64, (const void*)gest,
                               (const unsigned long long*)parts, pg, is_spin_glass, geo, key, gthr,
                               done, best_energy, best_index));
  } else {
    PQI_TRY(cudaLaunchKernelEx(&cfg, double_stream_kernel<float>, (const float*)w->W_f32z, w->ld, n,
                               theta, gains64, (const void*)gest,
                               (const unsigned long long*)parts, pg, is_spin_glass, geo, key, gthr,
                               done, best_energy, best_index));
  }
  PQI_LAUNCHED("double_stream_kernel");
  return PQI_OK;
}

pqi_status pqi_apply_flip(const pqi_weights* w, uint32_t* theta, double* gains64, int k, int l,
                          void* stream) {
  PQI_CHECK_ARG(w && theta && gains64 && k >= 0 && k < w->n && l < w->n && l != k);
  cudaStream_t s = as_stream(stream);
  const int grid = grid_for(w->n, 256, 148 * 4);
  if (w->kind == PQI_W_I8) {
    apply_flip_gains_kernel<int8_t><<<grid, 256, 0, s>>>(w->W_i8, w->ld, w->n, theta, gains64, k, l);
  } else {
    apply_flip_gains_kernel<float><<<grid, 256, 0, s>>>(w->W_f32z, w->ld, w->n, theta, gains64, k, l);
  }
  PQI_LAUNCHED("apply_flip_gains_kernel");
  toggle_bits_kernel<<<1, 1, 0, s>>>(theta, k, l);
  PQI_LAUNCHED("toggle_bits_kernel");
  return PQI_OK;
}

pqi_status pqi_rescore_fp64(const pqi_weights* w, const uint32_t* theta, int count, double* cut,
                            double* energy, void* workspace, size_t workspace_bytes,
                            void* stream) {
  PQI_CHECK_ARG(w && theta && count > 0 && (cut || energy));
  const int n = w->n, n32 = (n + 31) >> 5;
  const int nblk = std::max(1, std::min((n + 7) / 8, 2048));
  Workspace ws(workspace, workspace_bytes);
  double* partial = ws.take<double>((size_t)count * nblk * 2);
  PQI_CHECK_ARG(partial);
  cudaStream_t s = as_stream(stream);
  rescore_kernel<<<dim3(nblk, count), 256, 0, s>>>(w->W, n, theta, n32, partial);
  PQI_LAUNCHED("rescore_kernel");
  rescore_finish_kernel<<<(count + 127) / 128, 128, 0, s>>>(partial, nblk, count, cut, energy);
  PQI_LAUNCHED("rescore_finish_kernel");
  return PQI_OK;
}

pqi_status pqi_pack_bits(const uint8_t* bools, int rows, int n, uint32_t* words, void* stream) {
  PQI_CHECK_ARG(bools && words && rows > 0 && n > 0);
  const int n32 = (n + 31) >> 5;
  pack_kernel<<<grid_for((long long)rows * n32, 256), 256, 0, as_stream(stream)>>>(bools, rows, n,
                                                                                n32, words);
  PQI_LAUNCHED("pack_kernel");
  return PQI_OK;
}

pqi_status pqi_unpack_bits(const uint32_t* words, int rows, int n, uint8_t* bools, void* stream) {
  PQI_CHECK_ARG(bools && words && rows > 0 && n > 0);
  const int n32 = (n + 31) >> 5;
  unpack_kernel<<<grid_for((long long)rows * n, 256), 256, 0, as_stream(stream)>>>(words, rows, n,
                                                                                  n32, bools);
  PQI_LAUNCHED("unpack_kernel");
  return PQI_OK;
}

}  // extern "C"
