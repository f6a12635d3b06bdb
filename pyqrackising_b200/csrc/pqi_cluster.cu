// libpqi: steepest single-flip ascent of one state spread over a thread-block
// cluster (distributed shared memory), for low latency per flip on large n.
//
// A cluster of C CTAs runs one task (graph, starting state) at a time. CTA r
// owns nodes [r*S, r*S + S) (S = n / C rounded up to 32, so every 32-node bit
// word belongs to one CTA). Each thread owns NG groups of four nodes,
// lo + 4*(t + T*j) + i, and keeps their local fields y = W x and their bits in
// registers for the whole ascent.
//
// Per flip:
//   1. every thread applies the previous flip k to its fields
//      (y_v += coef * W_kv, one float4 / char4 of row k per group; the owner of
//      k toggles its bit) and folds the new gains g_v = x_v y_v into a local
//      argmax: float gain first, then the lowest node (a 64-bit key);
//   2. warp maxima (two 32-bit redux steps) meet in shared memory behind one
//      CTA barrier; warp 0 reduces them and lanes 0..C-1 write the CTA's best
//      (key, exact gain) into slot [rank] of every CTA with st.async, which
//      counts the bytes on that CTA's mbarrier;
//   3. thread 0 waits (bounded) for the C slots of the flip, a second CTA
//      barrier (which also spreads a failed wait) releases the CTA, and every
//      warp reduces the C local slots to the same global best, flipped next if
//      its gain is > 0.
// Two slot arrays and two mbarriers alternate between flips; a CTA can only be
// one flip ahead of any other, so a slot array is never rewritten while read.
// The selection rule is the batched kernel's (pqi_batch_search), so both give
// the same trajectory. Control flow depends only on values every CTA reads
// identically; the flip budget and the bounded waits end every loop.
#include <cooperative_groups.h>

#include <algorithm>
#include <type_traits>

#include "pqi_common.cuh"

namespace cg = cooperative_groups;

namespace pqi {

// Starting fields of the dense-graph tasks (pqi_batch.cu), freed by the caller.
pqi_status start_fields(const void* graphs, const int* task_graph, const uint32_t* init_states,
                        int words_pitch, int tasks, int max_n, bool i8, cudaStream_t s,
                        double** out, int* pitch);

struct ClusterGraph {  // same layout as the batched search's graph descriptor
  const void* W;
  int n;
  int ld;
  int kind;
  int pad;
  double upper_sum;
  const void* adj_ptr;  // row lists (unused here)
  const void* adj_col;
  const void* adj_val;
};

struct Slot {
  unsigned long long key;  // ord(float gain) << 32 | (0x3FFFFFFF - node) << 1 | bit
  double g;                // exact gain of that node
};

constexpr int kMaxCluster = 16;
constexpr long long kWaitCycles = 2000000000ll;  // ~1 s: a cluster peer that stops writing

__device__ __forceinline__ unsigned long long flip_key(float gv, int u, int xu) {
  return ((unsigned long long)ord_f32(gv) << 32) |
         (unsigned long long)(((0x3FFFFFFFu - (uint32_t)u) << 1) | (uint32_t)xu);
}

__device__ __forceinline__ int key_node(unsigned long long key) {
  return (int)(0x3FFFFFFFu - (((uint32_t)key) >> 1));
}

__device__ __forceinline__ float key_gain(unsigned long long key) {
  return unord_f32((uint32_t)(key >> 32));
}

// max of a 64-bit key over the warp: two 32-bit reductions (high word, then the
// low word among the lanes holding the highest high word)
__device__ __forceinline__ unsigned long long warp_max_key(unsigned long long key) {
  const uint32_t hi = __reduce_max_sync(0xFFFFFFFFu, (uint32_t)(key >> 32));
  const uint32_t lo =
      __reduce_max_sync(0xFFFFFFFFu, ((uint32_t)(key >> 32) == hi) ? (uint32_t)key : 0u);
  return ((unsigned long long)hi << 32) | lo;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

template <typename WT, int NG>
__global__ void __launch_bounds__(256) cluster_ascent_kernel(
    const ClusterGraph* __restrict__ graphs, const int* __restrict__ task_graph,
    const uint32_t* __restrict__ init_states, int words_pitch, int tasks, int spin,
    int flip_budget, uint32_t* __restrict__ best_states, double* __restrict__ best_values,
    unsigned long long* __restrict__ flips_total, int* __restrict__ status, double target,
    int* __restrict__ reached, const double* __restrict__ start_fields, int fields_pitch) {
  typedef typename std::conditional<sizeof(WT) == 1, int, double>::type GT;
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  extern __shared__ __align__(16) unsigned char smem[];
  // slots[p][r]: CTA r's best of the flips with parity p, written here by CTA r
  __shared__ __align__(16) Slot slots[2][kMaxCluster];
  __shared__ __align__(8) unsigned long long bar[2];
  __shared__ double qslot[kMaxCluster];
  __shared__ unsigned long long red_key[8];
  __shared__ double red_g[8];
  __shared__ int abort_flag;
  __shared__ int stop_flag;  // written by rank 0 (target mode)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int T = blockDim.x, nwarps = T >> 5;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  cl.sync();
  uint32_t phase = 0;  // bit p: parity of bar[p]'s current phase
  int par = 0;
  const int clusters = gridDim.x / C;
  for (int task = blockIdx.x / C; task < tasks; task += clusters) {
    const ClusterGraph G = graphs[task_graph[task]];
    const int n = G.n, n32 = (n + 31) >> 5;
    const WT* __restrict__ W = static_cast<const WT*>(G.W);
    const int S = (((n + C - 1) / C) + 31) & ~31;
    const int lo = rank * S, hi = min(n, lo + S);
    uint32_t* bits = reinterpret_cast<uint32_t*>(smem);
    GT* y0 = reinterpret_cast<GT*>(smem + (((size_t)n32 * 4 + 15) & ~size_t(15)));
    for (int w = threadIdx.x; w < n32; w += T) bits[w] = init_states[(size_t)task * words_pitch + w];
    __syncthreads();
    // starting local fields of the slice: computed beforehand for all tasks
    // (start_fields_kernel), else one warp per row
    if (start_fields && !G.adj_ptr) {
      const double* __restrict__ yrow = start_fields + (size_t)task * fields_pitch;
      for (int v = lo + (int)threadIdx.x; v < hi; v += T) y0[v - lo] = (GT)yrow[v];
    } else {
      for (int v = lo + warp; v < hi; v += nwarps) {
        const WT* row = W + (size_t)v * G.ld;
        GT acc = 0;
        for (int u = lane; u < n; u += 32) {
          const GT w = (GT)row[u];
          acc += ((bits[u >> 5] >> (u & 31)) & 1) ? w : -w;
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
        if (lane == 0) y0[v - lo] = acc;
      }
    }
    __syncthreads();
    GT y[4 * NG];
    uint32_t xm = 0;  // bit 4j+i: the bit of node lo + 4*(t + T*j) + i
    double qp = 0.0;
#pragma unroll
    for (int j = 0; j < NG; ++j)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int v = lo + 4 * ((int)threadIdx.x + T * j) + i;
        y[4 * j + i] = 0;
        if (v < hi) {
          y[4 * j + i] = y0[v - lo];
          const uint32_t b = (bits[v >> 5] >> (v & 31)) & 1;
          xm |= b << (4 * j + i);
          qp += b ? (double)y[4 * j + i] : -(double)y[4 * j + i];
        }
      }
    // q = sum_v x_v y_v over the cluster: partials stored into every CTA and
    // summed in rank order (the same double everywhere)
    for (int o = 16; o > 0; o >>= 1) qp += __shfl_xor_sync(0xFFFFFFFFu, qp, o);
    if (lane == 0) red_g[warp] = qp;
    __syncthreads();
    if ((int)threadIdx.x < C) {
      double a = 0.0;
      for (int i = 0; i < nwarps; ++i) a += red_g[i];
      *cl.map_shared_rank(&qslot[rank], (int)threadIdx.x) = a;
    }
    cl.sync();
    double q = 0.0;
    for (int r = 0; r < C; ++r) q += qslot[r];
    const double scale = spin ? 2.0 : 1.0;
    double val = spin ? -q / 2.0 : (2.0 * G.upper_sum - q) / 4.0;
    unsigned long long nflips = 0;
    int timeout = 0, failed = 0;
    int k = -1;
    GT coef = 0;
    for (int f = 0;; ++f) {
      if (k >= 0) {
        // apply the previous flip (node k) to my fields
        const WT* __restrict__ row = W + (size_t)k * G.ld;
        WT w[4 * NG];
#pragma unroll
        for (int j = 0; j < NG; ++j) {
          const int v = lo + 4 * ((int)threadIdx.x + T * j);
          if (v + 3 < n) {
            if constexpr (sizeof(WT) == 4) {
              const float4 t = __ldg(reinterpret_cast<const float4*>(row + v));
              w[4 * j] = t.x;
              w[4 * j + 1] = t.y;
              w[4 * j + 2] = t.z;
              w[4 * j + 3] = t.w;
            } else {
              const char4 t = __ldg(reinterpret_cast<const char4*>(row + v));
              w[4 * j] = t.x;
              w[4 * j + 1] = t.y;
              w[4 * j + 2] = t.z;
              w[4 * j + 3] = t.w;
            }
          } else {
#pragma unroll
            for (int i = 0; i < 4; ++i) w[4 * j + i] = (v + i < n) ? row[v + i] : (WT)0;
          }
        }
#pragma unroll
        for (int j = 0; j < 4 * NG; ++j) y[j] += coef * (GT)w[j];
        const int rel = k - lo;
        if (rel >= 0 && rel < S) {
          const int grp = rel >> 2;
          if (grp % T == (int)threadIdx.x) xm ^= 1u << (4 * (grp / T) + (rel & 3));
        }
      }
      // target mode: a task whose value reaches the target raises the global
      // flag; every 16 flips rank 0 reads it and hands it to the cluster's
      // CTAs behind a cluster barrier, so all of them stop at the same flip
      // (fields and bits then hold every accepted flip)
      if (reached && (f & 15) == 15) {
        if (rank == 0 && threadIdx.x == 0) {
          if (val >= target) atomicExch(reached, 1);
          const int r = *(volatile int*)reached;
          for (int c = 0; c < C; ++c) *cl.map_shared_rank(&stop_flag, c) = r;
        }
        cl.sync();
        if (stop_flag) break;
      }
      // my best flip: float gain first, then the lowest node (nodes ascend)
      float bv = -INFINITY;
      int bi = -1, bx = 0;
      double bg = 0.0;
#pragma unroll
      for (int j = 0; j < NG; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int v = lo + 4 * ((int)threadIdx.x + T * j) + i;
          if (v < hi) {
            const int xv = (xm >> (4 * j + i)) & 1;
            const double g = xv ? (double)y[4 * j + i] : -(double)y[4 * j + i];
            const float gv = (float)g;
            if (gv > bv) {  // strict: the lowest node keeps a tie
              bv = gv;
              bi = v;
              bg = g;
              bx = xv;
            }
          }
        }
      const unsigned long long key = bi >= 0 ? flip_key(bv, bi, bx) : 0ull;
      const unsigned long long wkey = warp_max_key(key);
      if (lane == 0) red_key[warp] = wkey;
      if (key != 0ull && key == wkey) red_g[warp] = bg;
      // arm this flip's barrier: C slots of 16 bytes are expected
      if (threadIdx.x == 0)
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                         smem_addr(&bar[par])),
                     "r"(C * (int)sizeof(Slot))
                     : "memory");
      __syncthreads();
      int bad = 0;
      if (warp == 0) {
        const unsigned long long ck = lane < nwarps ? red_key[lane] : 0ull;
        const double cgv = lane < nwarps ? red_g[lane] : 0.0;
        const unsigned long long cb = warp_max_key(ck);
        const uint32_t src = __ballot_sync(0xFFFFFFFFu, ck == cb && cb != 0ull);
        const double cbg = __shfl_sync(0xFFFFFFFFu, cgv, src ? __ffs(src) - 1 : 0);
        // the next row is one of the C CTAs' candidates: pull this CTA's
        // candidate row into L2 while the exchange is in flight (a hint only;
        // a row is ld * sizeof(WT) bytes, 16-byte aligned, inside W)
        if (lane == 0 && cb != 0ull && key_gain(cb) > 0.0f) {
          const WT* cand = W + (size_t)key_node(cb) * G.ld;
          asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(cand),
                       "r"((uint32_t)((size_t)G.ld * sizeof(WT)))
                       : "memory");
        }
        if (lane < C) {
          // this CTA's best into slot [rank] of CTA `lane`, counted on its bar[par]
          uint32_t raddr, rbar;
          asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                       : "=r"(raddr)
                       : "r"(smem_addr(&slots[par][rank])), "r"(lane));
          asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                       : "=r"(rbar)
                       : "r"(smem_addr(&bar[par])), "r"(lane));
          asm volatile(
              "st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.u64 [%0], {%1, %2}, "
              "[%3];" ::"r"(raddr),
              "l"(cb), "l"(__double_as_longlong(cbg)), "r"(rbar)
              : "memory");
        }
        if (lane == 0) {
          // wait (bounded) for the C slots of this flip
          const uint32_t ph = (phase >> par) & 1;
          const long long t0 = clock64();
          uint32_t done = 0;
          while (true) {
            asm volatile(
                "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                " selp.u32 %0, 1, 0, p;\n}"
                : "=r"(done)
                : "r"(smem_addr(&bar[par])), "r"(ph)
                : "memory");
            if (done || clock64() - t0 > kWaitCycles) break;
          }
          bad = !done;
        }
      }
      if (__syncthreads_or(bad)) {
        failed = 1;
        break;
      }
      phase ^= 1u << par;
      // the cluster's best (identical in every CTA)
      const unsigned long long sk = lane < C ? slots[par][lane].key : 0ull;
      const double sg = lane < C ? slots[par][lane].g : 0.0;
      const unsigned long long gkey = warp_max_key(sk);
      const uint32_t gsrc = __ballot_sync(0xFFFFFFFFu, sk == gkey && gkey != 0ull);
      const double gk = __shfl_sync(0xFFFFFFFFu, sg, gsrc ? __ffs(gsrc) - 1 : 0);
      par ^= 1;
      if (gkey == 0ull || !(key_gain(gkey) > 0.0f)) break;
      if (f >= flip_budget) {
        timeout = 1;
        break;
      }
      k = key_node(gkey);
      coef = (gkey & 1ull) ? (GT)-2 : (GT)2;
      val += scale * gk;
      ++nflips;
    }
    if (reached && rank == 0 && threadIdx.x == 0 && val >= target) atomicExch(reached, 1);
    // (the last accepted flip was applied by the pass that found no further one)
    // bits back to shared memory: eight lanes assemble one 32-node word
#pragma unroll
    for (int j = 0; j < NG; ++j) {
      const int v0 = lo + 4 * ((int)threadIdx.x + T * j);
      uint32_t wd = ((xm >> (4 * j)) & 15u) << (4 * (lane & 7));
      wd |= __shfl_xor_sync(0xFFFFFFFFu, wd, 1);
      wd |= __shfl_xor_sync(0xFFFFFFFFu, wd, 2);
      wd |= __shfl_xor_sync(0xFFFFFFFFu, wd, 4);
      if ((lane & 7) == 0 && v0 < hi) bits[v0 >> 5] = wd;
    }
    if (failed && threadIdx.x == 0) *cl.map_shared_rank(&abort_flag, 0) = 1;
    cl.sync();  // all slices final before rank 0 gathers the bits
    if (rank == 0) {
      for (int w = threadIdx.x; w < n32; w += T)
        best_states[(size_t)task * words_pitch + w] = *cl.map_shared_rank(&bits[w], (w * 32) / S);
      if (threadIdx.x == 0) {
        best_values[task] = val;
        atomicAdd(flips_total, nflips);
        if (timeout) atomicExch(status, PQI_ETIMEOUT);
      }
    }
    const int stop = *cl.map_shared_rank(&abort_flag, 0);
    cl.sync();  // no CTA starts the next task while another still reads its bits
    if (stop) {
      // a peer stopped answering: report and leave (every CTA read the flag)
      if (rank == 0 && threadIdx.x == 0) atomicExch(status, PQI_ETIMEOUT);
      return;
    }
  }
}

}  // namespace pqi

using namespace pqi;

extern "C" pqi_status pqi_cluster_ascent(const void* graphs, int num_graphs,
                                         const int* task_graph, const uint32_t* init_states,
                                         int words_pitch, int tasks, int max_n, int kind,
                                         int is_spin_glass, int cluster_size, int flip_budget,
                                         uint32_t* best_states, double* best_values,
                                         unsigned long long* flips_total, int* status,
                                         double target, int* reached, void* stream) {
  PQI_CHECK_ARG(graphs && num_graphs > 0 && task_graph && init_states && tasks > 0 && max_n > 0);
  PQI_CHECK_ARG(best_states && best_values && flips_total && status && flip_budget > 0);
  PQI_CHECK_ARG(cluster_size == 2 || cluster_size == 4 || cluster_size == 8 ||
                cluster_size == 16);
  PQI_CHECK_ARG(words_pitch >= (max_n + 31) / 32);
  PQI_CHECK_ARG(max_n < (1 << 30));
  const bool i8 = kind == PQI_W_I8;
  const int S = (((max_n + cluster_size - 1) / cluster_size) + 31) & ~31;
  // threads: one group of four nodes each where the slice allows, up to 256;
  // groups per thread (held in registers) rounded up to a power of two
  const int groups = (S + 3) / 4;
  const int T = std::max(32, std::min(256, (groups + 31) / 32 * 32));
  int NG = (groups + T - 1) / T;
  NG = NG <= 1 ? 1 : NG <= 2 ? 2 : NG <= 4 ? 4 : NG <= 8 ? 8 : 0;
  if (NG == 0) {
    set_error_text("cluster ascent: graph too large for this cluster size (use 16)");
    return PQI_EINVAL;
  }
  const size_t smem = (((size_t)((max_n + 31) >> 5) * 4 + 15) & ~size_t(15)) +
                      (size_t)S * (i8 ? sizeof(int) : sizeof(double));
  if (smem > 200 * 1024) {
    set_error_text("cluster ascent: slice does not fit in shared memory");
    return PQI_EINVAL;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.blockDim = dim3(T);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = as_stream(stream);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster_size;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const ClusterGraph* gd = static_cast<const ClusterGraph*>(graphs);
  // the starting fields of dense-graph tasks, one pass over W per task tile
  double* sf = nullptr;
  int sf_pitch = 0;
  {
    pqi_status r = start_fields(graphs, task_graph, init_states, words_pitch, tasks, max_n, i8,
                                as_stream(stream), &sf, &sf_pitch);
    if (r != PQI_OK) return r;
  }
  auto launch = [&](auto kern) -> pqi_status {
    PQI_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (cluster_size > 8)
      PQI_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    // as many clusters as fit at once; each loops over tasks (the occupancy
    // query is cached per kernel and launch shape: it is slow on first use)
    struct FitEntry {
      const void* k;
      size_t smem;
      int T, cs, dev, fit;
    };
    static FitEntry cache[32];
    static int cached = 0;
    int dev = 0;
    PQI_TRY(cudaGetDevice(&dev));
    int fit = 0;
    for (int e = 0; e < cached; ++e)
      if (cache[e].k == (const void*)kern && cache[e].smem == smem && cache[e].T == T &&
          cache[e].cs == cluster_size && cache[e].dev == dev)
        fit = cache[e].fit;
    if (fit == 0) {
      cfg.gridDim = dim3(cluster_size);
      PQI_TRY(cudaOccupancyMaxActiveClusters(&fit, kern, &cfg));
      if (fit > 0 && cached < 32) cache[cached++] = {(const void*)kern, smem, T, cluster_size, dev, fit};
    }
    if (fit < 1) {
      set_error_text("cluster ascent: the cluster does not fit on the device");
      return PQI_EINVAL;
    }
    const int clusters = std::max(1, std::min(tasks, fit));
    cfg.gridDim = dim3(clusters * cluster_size);
    PQI_TRY(cudaLaunchKernelEx(&cfg, kern, gd, task_graph, init_states, words_pitch, tasks,
                               is_spin_glass, flip_budget, best_states, best_values, flips_total,
                               status, target, reached, (const double*)sf, sf_pitch));
    return PQI_OK;
  };
  pqi_status st;
  if (i8) {
    st = NG == 1   ? launch(cluster_ascent_kernel<int8_t, 1>)
         : NG == 2 ? launch(cluster_ascent_kernel<int8_t, 2>)
         : NG == 4 ? launch(cluster_ascent_kernel<int8_t, 4>)
                   : launch(cluster_ascent_kernel<int8_t, 8>);
  } else {
    st = NG == 1   ? launch(cluster_ascent_kernel<float, 1>)
         : NG == 2 ? launch(cluster_ascent_kernel<float, 2>)
         : NG == 4 ? launch(cluster_ascent_kernel<float, 4>)
                   : launch(cluster_ascent_kernel<float, 8>);
  }
  if (st != PQI_OK) return st;
  PQI_LAUNCHED("cluster_ascent_kernel");
  if (sf) PQI_TRY(cudaFreeAsync(sf, as_stream(stream)));
  return PQI_OK;
}
