// Shared device/host helpers of libpqi (sm_100a).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <cmath>

#include "pqi.h"

namespace pqi {

// Last CUDA error seen by the library (host side, for diagnostics).
void set_error(cudaError_t e, const char* where);
void set_error_text(const char* msg);

#define PQI_TRY(expr)                                  \
  do {                                                 \
    cudaError_t e_ = (expr);                           \
    if (e_ != cudaSuccess) {                           \
      ::pqi::set_error(e_, #expr);                     \
      return PQI_ECUDA;                                \
    }                                                  \
  } while (0)

#define PQI_LAUNCHED(name)                             \
  do {                                                 \
    cudaError_t e_ = cudaGetLastError();               \
    if (e_ != cudaSuccess) {                           \
      ::pqi::set_error(e_, name);                      \
      return PQI_ECUDA;                                \
    }                                                  \
  } while (0)

#define PQI_CHECK_ARG(cond)         \
  do {                              \
    if (!(cond)) return PQI_EINVAL; \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ---------------------------------------------------------------------------
// Bump allocator over a caller-provided workspace (256-byte aligned slices).
struct Workspace {
  char* base;
  size_t size;
  size_t used;
  Workspace(void* p, size_t n) : base(static_cast<char*>(p)), size(n), used(0) {}
  template <typename T>
  T* take(size_t count) {
    size_t off = (used + 255) & ~size_t(255);
    size_t bytes = count * sizeof(T);
    if (!base || off + bytes > size) return nullptr;
    used = off + bytes;
    return reinterpret_cast<T*>(base + off);
  }
};

// ---------------------------------------------------------------------------
// Selection with the reference's tie-break.
//
// Item i of `count` belongs to work-item t = i % G at position j = i / G of that
// work-item's grid-stride sequence, in work-group grp = t / L at slot
// lane = t % L. The reference keeps, for equal values: the lowest group
// (host np.argmax), then the slot that wins the halving tree (rank[lane],
// computed on the host by replaying the tree; slots the tree never folds into
// slot 0 get rank 0xFF and are never selected), then the lowest j (strict '>'
// in the grid-stride loop). The 64-bit key orders items exactly that way:
//   high 32 bits: the float value mapped to an order-preserving unsigned
//   low 32 bits : ~priority, priority = ((grp * L + rank) * J + j)
// so the maximum key is the reference's selection. Key 0 = never selected.
struct SelGeom {
  uint32_t G, L, J;
  uint8_t rank[64];          // slot -> tie rank (0 wins), 0xFF: never reaches slot 0
  uint8_t slot_of_rank[64];  // inverse of rank
};

// Host: build the geometry for `count` items; false on an invalid geometry.
bool make_sel_geom(long count, int G, int L, SelGeom* out);

__host__ __device__ __forceinline__ uint32_t ord_f32(float v) {
#ifdef __CUDA_ARCH__
  uint32_t b = __float_as_uint(v);
#else
  uint32_t b;
  memcpy(&b, &v, 4);
#endif
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__host__ __device__ __forceinline__ float unord_f32(uint32_t o) {
  uint32_t b = (o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o;
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  float f;
  memcpy(&f, &b, 4);
  return f;
#endif
}

__host__ __device__ __forceinline__ uint64_t sel_key(float v, uint64_t i, const SelGeom& g) {
  if (v != v) return 0ull;  // NaN: the reference's strict '>' never takes it
  const uint32_t t = (uint32_t)(i % g.G);
  const uint32_t j = (uint32_t)(i / g.G);
  const uint32_t grp = t / g.L;
  const uint32_t r = g.rank[t - grp * g.L];
  if (r == 0xFFu) return 0ull;
  const uint32_t pr = (grp * g.L + r) * g.J + j;
  return ((uint64_t)ord_f32(v) << 32) | (uint64_t)(0xFFFFFFFFu - pr);
}

__host__ __device__ __forceinline__ void sel_decode(uint64_t key, const SelGeom& g, float* v,
                                                    int64_t* idx) {
  if (key == 0ull) {
    *v = -INFINITY;
    *idx = -1;
    return;
  }
  *v = unord_f32((uint32_t)(key >> 32));
  const uint32_t pr = 0xFFFFFFFFu - (uint32_t)(key & 0xFFFFFFFFu);
  const uint32_t j = pr % g.J;
  const uint32_t gr = pr / g.J;
  const uint32_t grp = gr / g.L;
  const uint32_t r = gr - grp * g.L;
  const uint32_t t = grp * g.L + g.slot_of_rank[r];
  *idx = (int64_t)t + (int64_t)j * g.G;
}

__device__ __forceinline__ uint64_t warp_max_u64(uint64_t k) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    uint64_t other = __shfl_xor_sync(0xFFFFFFFFu, k, o);
    k = other > k ? other : k;
  }
  return k;
}

// Block-wide max of a u64 key; every thread gets the result. `scratch` holds
// >= 32 u64. Contains two __syncthreads().
__device__ __forceinline__ uint64_t block_max_u64(uint64_t k, uint64_t* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
  k = warp_max_u64(k);
  if (lane == 0) scratch[warp] = k;
  __syncthreads();
  uint64_t r = lane < nwarps ? scratch[lane] : 0ull;
  r = warp_max_u64(r);
  __syncthreads();
  return r;
}

// Bits: node j of a 32-bit-word string.
__device__ __forceinline__ int get_bit32(const uint32_t* w, uint32_t j) {
  return (w[j >> 5] >> (j & 31)) & 1u;
}

__host__ __device__ __forceinline__ long long pair_base(long long k, long long n) {
  // linear index of pair (k, k+1) in the reference's k-major enumeration
  return k * (n - 1) - (k * (k - 1)) / 2;
}

// Launch helpers shared across translation units (pqi_core.cu).
pqi_status launch_gains(const pqi_weights* w, const uint32_t* theta, int count, float* g32,
                        double* g64, cudaStream_t s);
pqi_status launch_select(const float* vals, long long count, float scale, const SelGeom& geo,
                         unsigned long long* key, float* best_val, int* best_idx,
                         cudaStream_t s);

}  // namespace pqi
