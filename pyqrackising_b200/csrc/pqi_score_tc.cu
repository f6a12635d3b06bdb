// libpqi: tensor-core (tcgen05) batched scoring for sm_100a.
//
// Y = X W for a batch of candidates X (B x n, entries +-1) and the coupling
// matrix W (n x n, symmetric, zero diagonal), then q_b = sum_j x_bj Y_bj in the
// epilogue (score_finish in pqi_score.cu turns q into the reference's value).
//
//  * int8 path (integer weights in [-127, 127]): A = X as int8 +-1, B = W_i8,
//    kind::i8 MMAs with int32 accumulation: exact.
//  * float path: W = hi + lo (two bf16 matrices), A = X as bf16 +-1, two K
//    passes (hi then lo) into one float32 accumulator (kind::f16).
//
// A persistent CTA per SM walks 128 x 256 tiles of Y (candidates x nodes),
// each over all of K, with a 4-stage shared-memory ring and two 256-column
// TMEM accumulators so the epilogue of one tile overlaps the MMAs of the next:
//   warp 0    : TMA loads of the +-1 candidate tile (expanded from the packed
//               bits by a short pass, L2-resident) and of the W tile (W is
//               symmetric, so its rows are the K-major rows the B operand
//               needs); ragged edges come from the TMA zero fill
//   warp 1    : TMEM allocation; lane 0 issues tcgen05.mma
//   warps 2-5 : epilogue: tcgen05.ld, row-dot with x, one partial per row;
//               the last tile of a candidate block folds the block into the
//               reference-order selection (no separate finish launch)
// Every mbarrier wait is bounded by a clock budget; on expiry the CTA records
// an error, the outputs become NaN / index -1, and TMEM is still released.
#include <cuda.h>

#include <algorithm>

#include <cooperative_groups.h>

#include "pqi_common.cuh"
#include "pqi_tc.cuh"

namespace pqi {

namespace tc {

constexpr int BM = 128;           // candidates per tile (UMMA M)
constexpr int BN = 256;           // nodes per tile (UMMA N)
constexpr int BK_BYTES = 128;     // K bytes per stage (one 128-byte swizzle row)
constexpr int STAGES = 4;
constexpr int A_STAGE = BM * BK_BYTES;   // 16 KB
constexpr int B_STAGE = BN * BK_BYTES;   // 32 KB
constexpr int STAGE_BYTES = A_STAGE + B_STAGE;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;  // + alignment slack
// CTA-pair mode (cta_group::2): a pair computes 256 candidates x 256 nodes
// with M = 256 MMAs issued by the even CTA; each CTA loads its 128 candidate
// rows and half (128 rows) of the W tile, so each CTA's W traffic halves.
constexpr int B_STAGE_PAIR = (BN / 2) * BK_BYTES;  // 16 KB
constexpr int STAGE_BYTES_PAIR = A_STAGE + B_STAGE_PAIR;
constexpr int STAGES_PAIR = 6;
constexpr int MAX_STAGES = STAGES_PAIR;
static_assert(STAGES_PAIR * STAGE_BYTES_PAIR + 1024 <= SMEM_BYTES, "pair ring fits the same smem");
constexpr uint32_t kPeerMask = 0xFEFFFFFFu;  // clears the pair bit of a shared::cluster address

// Instruction descriptors (M = 128, N = 256, both operands K-major).
constexpr uint32_t kIdescI8 = (2u << 4)      // D: s32
                              | (1u << 7)    // A: signed int8
                              | (1u << 10)   // B: signed int8
                              | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
constexpr uint32_t kIdescBF16 = (1u << 4)    // D: f32
                                | (1u << 7)  // A: bf16
                                | (1u << 10) // B: bf16
                                | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

constexpr uint32_t kIdescI8Pair = (kIdescI8 & ~(0x1Fu << 24)) | ((uint32_t)(256 >> 4) << 24);
constexpr uint32_t kIdescBF16Pair = (kIdescBF16 & ~(0x1Fu << 24)) | ((uint32_t)(256 >> 4) << 24);

// Warp roles of the persistent kernel (6 warps, 10 when the A operand is
// expanded in the kernel).
constexpr int TMA_WARP = 0;       // warp 0 lane 0: TMA loads of the W (and X) tiles
constexpr int MMA_WARP = 1;       // warp 1: TMEM alloc, lane 0 issues MMAs
constexpr int PTHREADS = 192;     // warps 2-5: epilogue (TMEM lane quarter = warp % 4)
constexpr int FTHREADS = 320;     // + warps 6-9: A-operand producers (FUSED)
constexpr int ACC_COLS = 512;     // two 256-column accumulators
// FUSED: each producer thread owns one A row; the packed bits it needs run
// PF stages ahead through a per-thread cp.async ring in shared memory
// (16 bytes per stage: four words of int8 columns, two of bf16 columns).
constexpr int PF = 6;
constexpr int PF_BYTES = PF * 128 * 16;  // 12 KB
constexpr int SMEM_BYTES_FUSED = STAGES * STAGE_BYTES + PF_BYTES + 1024;
static_assert(SMEM_BYTES_FUSED <= 227 * 1024, "fused ring fits");

__device__ __forceinline__ void epi_barrier() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Persistent scoring kernel: CTA c handles the contiguous tiles
// [c * T / grid, (c + 1) * T / grid); tile t covers candidates
// [128 * (t / ntn), +128) x nodes [256 * (t % ntn), +256). A CTA that owns a
// whole candidate block keeps q in registers across its node tiles; a block
// split between two CTAs goes through per-tile partials summed in tile order
// by the CTA that completes it. The finisher converts q to the reference's
// value and folds it into the selection key; the last block decodes it.
// One packed word (32 columns) of a candidate -> the A operand's 16-byte
// chunks: int8 +-1 (32 bytes = two chunks) or bf16 +-1 (64 bytes = four
// chunks); bit set = +1.
__device__ __forceinline__ void pm1_i8x4(uint32_t nib, uint32_t& o) {
  // four bits -> four bytes 0x01 (set) / 0xFF (clear)
  const uint32_t t = ((nib & 0xFu) * 0x00204081u) & 0x01010101u;
  o = 0xFFFFFFFFu - t * 0xFEu;
}

__device__ __forceinline__ uint32_t pm1_bf16x2(uint32_t two) {
  // two bits -> two bf16: 0x3F80 (+1) / 0xBF80 (-1)
  const uint32_t nb = ~two;
  return 0x3F803F80u | ((nb & 1u) << 15) | ((nb & 2u) << 30);
}

__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src),
               "r"(valid ? 4 : 0)
               : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <bool kInt8, bool PAIR, bool FUSED>
__global__ void __launch_bounds__(FUSED ? FTHREADS : PTHREADS, 1)
    score_tc_kernel(const __grid_constant__ CUtensorMap map_a,
                    const __grid_constant__ CUtensorMap map_b0,
                    const __grid_constant__ CUtensorMap map_b1,
                    const __grid_constant__ CUtensorMap map_b2,
                    const __grid_constant__ CUtensorMap map_b3, int planes, double qscale,
                    int n, int shots,
                    const uint32_t* __restrict__ theta, int n32, double upper_sum, int spin,
                    SelGeom geo, double* __restrict__ qpart, float* __restrict__ energies,
                    unsigned int* __restrict__ mcount, unsigned int* __restrict__ mdone,
                    unsigned long long* __restrict__ key, float* __restrict__ best_energy,
                    int* __restrict__ best_index, int* __restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[MAX_STAGES];
  __shared__ __align__(8) uint64_t empty_bar[MAX_STAGES];
  __shared__ __align__(8) uint64_t accf_bar[2];
  __shared__ __align__(8) uint64_t acce_bar[2];
  __shared__ uint32_t tmem_base_holder;
  __shared__ int s_fail;
  __shared__ unsigned int s_bcast;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + ((1024 - (raw & 1023)) & 1023);

  // pair mode: ranks 0 (issues the MMAs) and 1 of a 2-CTA cluster; a unit of
  // work is the pair, a tile covers 256 candidates (128 per CTA)
  constexpr int NST = PAIR ? STAGES_PAIR : STAGES;
  constexpr int SB = PAIR ? STAGE_BYTES_PAIR : STAGE_BYTES;
  constexpr int UM = PAIR ? 2 * BM : BM;  // candidates per tile
  const int rank = PAIR ? (int)(blockIdx.x & 1) : 0;
  const int unit = PAIR ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
  const int units = PAIR ? (int)(gridDim.x >> 1) : (int)gridDim.x;
  const int ntn = (n + BN - 1) / BN;
  const int ntm = (shots + BM - 1) / BM;       // 128-candidate blocks (finish bookkeeping)
  const int ntu = (shots + UM - 1) / UM;       // tile rows
  const int ntiles = ntn * ntu;
  // each unit walks one contiguous chunk of tiles (candidate-block major), so
  // most blocks are finished by one unit with q kept in registers
  const int t_begin = (int)(((long long)unit * ntiles) / units);
  const int t_end = (int)(((long long)(unit + 1) * ntiles) / units);
  const int kb_per_pass = kInt8 ? (n + BK_BYTES - 1) / BK_BYTES : (n + 63) / 64;
  // int8 operands: `planes` K passes, each its own accumulation (planes = 4:
  // the digit planes of float weights, combined exactly in the epilogue);
  // bf16: the hi and lo passes accumulate into one accumulator
  const int upt = kInt8 ? planes : 1;                       // accumulations per tile
  const int spu = kInt8 ? kb_per_pass : 2 * kb_per_pass;    // stages per accumulation
  const int kblocks = upt * spu;                            // stages per tile

  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; ++s) {
      // FUSED: the W tile's TMA arrival plus one arrival per producer warp
      mbar_init(&full_bar[s], FUSED ? 5 : 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&accf_bar[a], 1);
      mbar_init(&acce_bar[a], PAIR ? 8 : 4);  // pair: both CTAs' epilogue warps
    }
    s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == MMA_WARP) {
    if constexpr (PAIR) {
      // both CTAs' warp 1, same destination: the pair's TMEM columns
      asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                       smem_u32(&tmem_base_holder)),
                   "r"(ACC_COLS));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    } else {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                       smem_u32(&tmem_base_holder)),
                   "r"(ACC_COLS));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  if constexpr (PAIR) {
    cooperative_groups::this_cluster().sync();  // both CTAs' barriers initialised
  } else {
    __syncthreads();
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem_base = tmem_base_holder;

  if (warp == TMA_WARP) {
    if (lane == 0) {
      uint32_t it = 0;
      bool ok = true;
      for (int t = t_begin; t < t_end && ok; ++t) {
        const int m0 = (t / ntn) * UM + rank * BM, n0 = (t % ntn) * BN + rank * (BN / 2);
        int kp = 0, pass = 0;  // K block within its pass, pass (plane, or hi / lo)
        for (int kb = 0; kb < kblocks; ++kb, ++it) {
          const int s = it % NST;
          if (it >= NST && !mbar_wait(&empty_bar[s], ((it / NST) - 1) & 1)) {
            ok = false;
            s_fail = 1;
            break;
          }
          const int kk = kInt8 ? kp * BK_BYTES : kp * 64;
          const CUtensorMap* mb =
              pass == 0 ? &map_b0 : (pass == 1 ? &map_b1 : (pass == 2 ? &map_b2 : &map_b3));
          if (++kp == kb_per_pass) {
            kp = 0;
            ++pass;
          }
          uint8_t* dst = smem + s * SB;
          if constexpr (PAIR) {
            // both CTAs' bytes count on the even CTA's barrier, armed there
            if (rank == 0) mbar_expect_tx(&full_bar[s], 2 * SB);
            const uint32_t bar = smem_u32(&full_bar[s]) & kPeerMask;
            tma_load_2d_pair(dst, &map_a, bar, kk, m0);
            tma_load_2d_pair(dst + A_STAGE, mb, bar, kk, n0);
          } else if constexpr (FUSED) {
            mbar_expect_tx(&full_bar[s], B_STAGE);  // the producers write the A tile
            tma_load_2d(dst + A_STAGE, mb, &full_bar[s], kk, n0);
          } else {
            mbar_expect_tx(&full_bar[s], STAGE_BYTES);
            tma_load_2d(dst, &map_a, &full_bar[s], kk, m0);
            tma_load_2d(dst + A_STAGE, mb, &full_bar[s], kk, n0);
          }
        }
      }
    }
    __syncwarp();
  } else if (warp == MMA_WARP) {
    if (lane == 0 && rank == 0) {  // pair: the even CTA issues for both
      const uint32_t idesc = PAIR ? (kInt8 ? kIdescI8Pair : kIdescBF16Pair)
                                  : (kInt8 ? kIdescI8 : kIdescBF16);
      uint32_t it = 0;
      int i = 0;
      bool ok = true;
      const int units_total = (t_end - t_begin) * upt;
      for (int u = 0; u < units_total && ok; ++u, ++i) {
        const int a = i & 1;
        if (i >= 2 && !mbar_wait(&acce_bar[a], ((i >> 1) - 1) & 1)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tmem_d = tmem_base + (uint32_t)(a * BN);
        for (int kb = 0; kb < spu; ++kb, ++it) {
          const int s = it % NST;
          if (!mbar_wait(&full_bar[s], (it / NST) & 1)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a_addr = smem_u32(smem + s * SB);
          const uint32_t b_addr = a_addr + A_STAGE;
#pragma unroll
          for (int k = 0; k < BK_BYTES / 32; ++k) {
            if constexpr (PAIR) {
              mma_pair<kInt8>(tmem_d, sw128_desc(a_addr + k * 32), sw128_desc(b_addr + k * 32),
                              idesc, (kb > 0 || k > 0) ? 1u : 0u);
            } else {
              mma<kInt8>(tmem_d, sw128_desc(a_addr + k * 32), sw128_desc(b_addr + k * 32), idesc,
                         (kb > 0 || k > 0) ? 1u : 0u);
            }
          }
          // frees the stage (in both CTAs of a pair) once these MMAs have read it
          if constexpr (PAIR) {
            mma_commit_pair(&empty_bar[s]);
          } else {
            mma_commit(&empty_bar[s]);
          }
        }
        if (ok) {  // accumulator a complete
          if constexpr (PAIR) {
            mma_commit_pair(&accf_bar[a]);
          } else {
            mma_commit(&accf_bar[a]);
          }
        }
      }
      if (!ok) s_fail = 1;
    }
    __syncwarp();
  } else if (FUSED && warp >= 6) {
    // ---- A producers: warps 6-9, thread p writes row p of every A tile ----
    // Stages run tile by tile, kblocks per tile, K blocks within each pass in
    // order. The row's packed words for stage it + PF are copied into
    // the thread's ring slot while stage it is expanded, so the L2 latency of
    // the bits is hidden behind PF stages of MMAs.
    const int p = threadIdx.x - 192;
    constexpr int WPS = kInt8 ? 4 : 2;  // packed words per stage
    const int nstage = (t_end - t_begin) * kblocks;
    // ring slot layout [slot][word q][thread p]: a warp's copies of one word
    // fall on 32 consecutive banks
    const uint32_t ring = smem_u32(smem + NST * SB) + (uint32_t)p * 4u;
    // the stage being prefetched: tile ti, K block ki, ring slot si (all
    // advanced by one per issue, no divisions in the loop)
    int ti = t_begin, ki = 0, kp = 0, si = 0, issued = 0;
    int tm_i = t_begin / ntn, tn_i = t_begin - (t_begin / ntn) * ntn;  // tile row / column of ti
    auto issue = [&]() {
      if (issued < nstage) {
        const int b = tm_i * BM + p;
        const int w0 = kp * (kInt8 ? 4 : 2);  // the stage's first word within the row
        const uint32_t* src = theta + (size_t)(b < shots ? b : 0) * n32;
        const uint32_t dst = ring + (uint32_t)si * (128u * 16u);
#pragma unroll
        for (int q = 0; q < WPS; ++q)
          cp_async4(dst + 512u * q, src + min(w0 + q, n32 - 1), b < shots && w0 + q < n32);
        if (++kp == kb_per_pass) kp = 0;
        if (++ki == kblocks) {
          ki = 0;
          kp = 0;
          ++ti;
          if (++tn_i == ntn) {
            tn_i = 0;
            ++tm_i;
          }
        }
        ++issued;
      }
      cp_async_commit();  // an empty group past the end keeps the count uniform
      if (++si == PF) si = 0;
    };
#pragma unroll 1
    for (int q = 0; q < PF; ++q) issue();
    bool ok = true;
    int slot_i = 0, s = 0;
    uint32_t phase = 0;  // parity of the ring pass of stage s
#pragma unroll 1
    for (int st = 0; st < nstage; ++st) {
      cp_async_wait<PF - 1>();  // this stage's words have landed
      uint32_t wd[4];
      const uint8_t* slot = smem + NST * SB + (size_t)p * 4 + (size_t)slot_i * (128 * 16);
#pragma unroll
      for (int q = 0; q < 4; ++q) wd[q] = (q < WPS) ? *reinterpret_cast<const volatile uint32_t*>(slot + 512 * q) : 0u;
      if (++slot_i == PF) slot_i = 0;
      issue();
      if (st >= NST && !mbar_wait_warp(&empty_bar[s], phase ^ 1u)) {
        ok = false;
        s_fail = 1;
      }
      if (__all_sync(0xFFFFFFFFu, ok)) {
        // row p of the 128-byte-swizzled K-major tile: 16-byte chunk c sits at
        // (c ^ (p & 7)) * 16 in the row
        uint8_t* rowp = smem + s * SB + p * BK_BYTES;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          uint32_t o[4];
          if constexpr (kInt8) {
            const uint32_t bits16 = (wd[c >> 1] >> ((c & 1) * 16)) & 0xFFFFu;
#pragma unroll
            for (int e = 0; e < 4; ++e) pm1_i8x4(bits16 >> (4 * e), o[e]);
          } else {
            const uint32_t bits8 = (wd[c >> 2] >> ((c & 3) * 8)) & 0xFFu;
#pragma unroll
            for (int e = 0; e < 4; ++e) o[e] = pm1_bf16x2(bits8 >> (2 * e));
          }
          *reinterpret_cast<uint4*>(rowp + ((c ^ (p & 7)) << 4)) = make_uint4(o[0], o[1], o[2], o[3]);
        }
        // generic-proxy writes -> visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      }
      __syncwarp();
      if (!__all_sync(0xFFFFFFFFu, ok)) break;
      if (lane == 0) mbar_arrive(&full_bar[s]);
      if (++s == NST) {
        s = 0;
        phase ^= 1u;
      }
    }
    cp_async_wait<0>();
  } else {
    // ---- epilogue: warps 2-5, all 128 threads take every branch together ----
    const int quarter = warp & 3;
    const int row = quarter * 32 + lane;
    // q of this thread's candidate over the CTA's tiles of the current block
    long long qacc_i = 0;
    double qacc_f = 0.0;
    int i = 0;
    for (int t = t_begin; t < t_end; ++t) {
      const int tm = t / ntn, tn = t % ntn;                // tile row, node tile
      const int tm128 = tm * (PAIR ? 2 : 1) + rank;          // this CTA's 128-candidate block
      const int b = tm128 * BM + row, n0 = tn * BN;
      // this CTA's share of candidate block tm: whole, or split with a neighbour
      const int blk0 = tm * ntn;
      const int first = max(t_begin, blk0), last = min(t_end, blk0 + ntn) - 1;
      const bool whole = first == blk0 && last == blk0 + ntn - 1;
      // candidate bits of this tile (independent of the MMAs: load before waiting)
      uint32_t xbits[BN / 32];
      {
        const uint32_t* th = theta + (size_t)(b < shots ? b : 0) * n32;
#pragma unroll
        for (int c = 0; c < BN / 32; ++c) {
          const int j0 = n0 + 32 * c;
          xbits[c] = (b < shots && j0 < n) ? __ldg(th + (j0 >> 5)) : 0u;
        }
      }
      // the tile's q over its accumulations (digit planes: sum_p q_p 2^(8(P-1-p)),
      // exact in 64 bits)
      long long qt_i = 0;
      double qt_f = 0.0;
      for (int pl = 0; pl < upt; ++pl, ++i) {
      const int a = i & 1;
      // columns beyond n hold zeros (TMA zero fill of W), so no column mask
      const bool ready = mbar_wait_warp(&accf_bar[a], (i >> 1) & 1);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (__all_sync(0xFFFFFFFFu, ready)) {
        const uint32_t tbase =
            tmem_base + (uint32_t)(a * BN) + ((uint32_t)(quarter * 32) << 16);
        // rounds of RC columns, the next round's load in flight while one is
        // summed (64 columns for int8, 32 for float)
        constexpr int RC = kInt8 ? 64 : 32;
        uint32_t r0[RC], r1[RC];
#pragma unroll
        for (int h = 0; h < RC / 32; ++h)
          tmem_load32_nowait(tbase + 32 * h, *reinterpret_cast<uint32_t(*)[32]>(&r0[32 * h]));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int h = 0; h < RC / 32; ++h) reg_fence32(*reinterpret_cast<uint32_t(*)[32]>(&r0[32 * h]));
        // int8: sum_j Y_bj and the sum over x_bj = +1 (|Y| <= 127 n, so 256
        // columns stay below 2^31 for n <= 65536, the int8 path's limit)
        int s_all = 0, s_set = 0;
        double f_q = 0.0;                 // float: sum_j x_bj Y_bj
#pragma unroll
        for (int rd = 0; rd < BN / RC; ++rd) {
          uint32_t(&cur)[RC] = (rd & 1) ? r1 : r0;
          uint32_t(&nxt)[RC] = (rd & 1) ? r0 : r1;
          if (rd + 1 < BN / RC) {
#pragma unroll
            for (int h = 0; h < RC / 32; ++h)
              tmem_load32_nowait(tbase + (uint32_t)(RC * (rd + 1) + 32 * h),
                                 *reinterpret_cast<uint32_t(*)[32]>(&nxt[32 * h]));
          }
#pragma unroll
          for (int h = 0; h < RC / 32; ++h) {
            const uint32_t xb = xbits[(RC / 32) * rd + h];
            if constexpr (kInt8) {
#pragma unroll
              for (int e = 0; e < 32; ++e) {
                const uint32_t v = cur[32 * h + e];
                const uint32_t m = 0u - ((xb >> e) & 1u);  // all ones where x_bj = +1
                s_all += (int)v;
                s_set += (int)(v & m);
              }
            } else {
              // x_bj Y_bj (sign bit flipped where x_bj = -1), summed pairwise in
              // float over the 32 columns, then added in double
              float t[16];
#pragma unroll
              for (int e = 0; e < 16; ++e) {
                const uint32_t s0 = ((xb >> (2 * e)) & 1u) ? 0u : 0x80000000u;
                const uint32_t s1 = ((xb >> (2 * e + 1)) & 1u) ? 0u : 0x80000000u;
                t[e] = __uint_as_float(cur[32 * h + 2 * e] ^ s0) +
                       __uint_as_float(cur[32 * h + 2 * e + 1] ^ s1);
              }
#pragma unroll
              for (int w = 8; w > 0; w >>= 1)
#pragma unroll
                for (int e = 0; e < w; ++e) t[e] = t[e] + t[e + w];
              f_q += (double)t[0];
            }
          }
          if (rd + 1 < BN / RC) {
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int h = 0; h < RC / 32; ++h)
              reg_fence32(*reinterpret_cast<uint32_t(*)[32]>(&nxt[32 * h]));
          }
        }
        // int8: sum_j x_bj Y_bj = 2 * (sum over x = +1) - (sum over all)
        if constexpr (kInt8) {
          qt_i += (2ll * (long long)s_set - (long long)s_all) << (8 * (upt - 1 - pl));
        } else {
          qt_f += f_q;
        }
      } else {
        s_fail = 1;
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) {  // accumulator a may be overwritten
        if (PAIR && rank == 1) {
          mbar_arrive_remote0(&acce_bar[a]);  // the even CTA issues the MMAs
        } else {
          mbar_arrive(&acce_bar[a]);
        }
      }
      }  // accumulations of the tile
      bool finish = false;  // this CTA folds block tm into the selection
      double q = 0.0;
      if (whole) {
        qacc_i += qt_i;
        qacc_f += qt_f;
        if (t == last) {
          finish = tm128 < ntm;  // (a pair's odd half can lie wholly past the batch)
          q = kInt8 ? (double)qacc_i * qscale : qacc_f;
          qacc_i = 0;
          qacc_f = 0.0;
        }
      } else {
        // split block: per-tile partials, summed in tile order by the CTA that
        // completes the block's tile count
        if (b < shots) qpart[(size_t)tn * shots + b] = kInt8 ? (double)qt_i : qt_f;
        if (t == last && tm128 < ntm) {  // (a pair's odd half can lie wholly past the batch)
          __threadfence();
          epi_barrier();
          if (quarter == 0 && lane == 0)
            s_bcast = atomicAdd(&mcount[tm128], (unsigned)(last - first + 1)) +
                      (unsigned)(last - first + 1);
          epi_barrier();
          if (s_bcast == (unsigned)ntn) {
            __threadfence();
            finish = true;
            if (b < shots) {
              for (int u = 0; u < ntn; ++u) q += __ldcg(qpart + (size_t)u * shots + b);
              if constexpr (kInt8) q *= qscale;
            }
          }
          epi_barrier();  // s_bcast is rewritten by a later block
        }
      }
      if (finish) {
        uint64_t kbest = 0;
        if (b < shots) {
          const double val = spin ? -q / 2.0 : (2.0 * upper_sum - q) / 4.0;
          const float v = (float)val;
          if (energies) energies[b] = v;
          kbest = sel_key(v, (uint64_t)b, geo);
        }
        kbest = warp_max_u64(kbest);
        if (lane == 0 && kbest) atomicMax(key, (unsigned long long)kbest);
        __threadfence();
        epi_barrier();
        if (quarter == 0 && lane == 0) {
          const unsigned done = atomicAdd(mdone, 1u);
          if (done == (unsigned)(ntm - 1)) {
            __threadfence();
            float v;
            int64_t idx;
            sel_decode(atomicAdd(key, 0ull), geo, &v, &idx);
            if (atomicAdd(err, 0) || s_fail) {
              v = __int_as_float(0x7FC00000);
              idx = -1;
            }
            if (best_energy) *best_energy = v;
            if (best_index) *best_index = (int)idx;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  if constexpr (PAIR) {
    // both CTAs done: no MMA writes the peer's TMEM, no arrival targets the
    // even CTA's barriers, before either releases TMEM or exits
    cooperative_groups::this_cluster().sync();
  } else {
    __syncthreads();
  }
  if (warp == MMA_WARP) {
    if constexpr (PAIR) {
      asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                   "r"(ACC_COLS));
    } else {
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                   "r"(ACC_COLS));
    }
  }
  if (threadIdx.x == 0 && s_fail) atomicExch(err, 1);
}

// One packed word -> 32 +-1 elements of the A operand.
template <typename T>
__device__ __forceinline__ void expand_word(uint32_t bits, T* __restrict__ dst) {
  if constexpr (sizeof(T) == 1) {
    // bit -> byte 0x01 (set) or 0xFF (clear), four at a time
    uint32_t o[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const uint32_t t = (((bits >> (4 * q)) & 0xFu) * 0x00204081u) & 0x01010101u;
      o[q] = 0xFFFFFFFFu - t * 0xFEu;
    }
    reinterpret_cast<uint4*>(dst)[0] = make_uint4(o[0], o[1], o[2], o[3]);
    reinterpret_cast<uint4*>(dst)[1] = make_uint4(o[4], o[5], o[6], o[7]);
  } else {
    uint32_t o[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const uint32_t lo = ((bits >> (2 * q)) & 1u) ? 0x3F80u : 0xBF80u;
      const uint32_t hi = ((bits >> (2 * q + 1)) & 1u) ? 0x3F80u : 0xBF80u;
      o[q] = lo | (hi << 16);
    }
    uint4* d4 = reinterpret_cast<uint4*>(dst);
#pragma unroll
    for (int q = 0; q < 4; ++q) d4[q] = make_uint4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
  }
}

// Packed candidates -> the +-1 A operand (int8, or bf16 for the float path),
// row pitch ld elements: one word per thread, so a warp's stores cover
// contiguous 32-byte (int8) or 64-byte (bf16) pieces of a row. Columns at and
// beyond n are never read (the A tensor map ends at n).
template <typename T>
__global__ void expand_pm1_kernel(const uint32_t* __restrict__ theta, int shots, int n32, int ld,
                                  T* __restrict__ X) {
  const long long total = (long long)shots * n32;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(e / n32), w = (int)(e - (long long)b * n32);
    expand_word<T>(__ldg(theta + e), X + (size_t)b * ld + (size_t)w * 32);
  }
}

}  // namespace tc


EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// 2-D K-major map: rows x cols elements (cols contiguous, row pitch `pitch`
// elements), box = box_rows x (128 bytes of elements), 128-byte swizzle.
static bool make_map(CUtensorMap* map, const void* base, bool int8, int rows, int cols, int pitch,
                     int box_rows) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return false;
  const int esz = int8 ? 1 : 2;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)pitch * esz};
  cuuint32_t box[2] = {(cuuint32_t)(128 / esz), (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, int8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                   const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}


struct MapCacheEntry {
  const void* base;
  int rows, cols, pitch, box_rows;
  bool int8;
  CUtensorMap map;
};

// Tensor maps depend only on (address, shape): keep the last few encoded.
bool cached_map(CUtensorMap* out, const void* base, bool int8, int rows, int cols, int pitch,
                int box_rows) {
  static MapCacheEntry cache[8] = {};
  static int next = 0;
  for (const auto& e : cache) {
    if (e.base == base && e.rows == rows && e.cols == cols && e.pitch == pitch &&
        e.box_rows == box_rows && e.int8 == int8) {
      *out = e.map;
      return true;
    }
  }
  MapCacheEntry e{base, rows, cols, pitch, box_rows, int8, {}};
  if (!make_map(&e.map, base, int8, rows, cols, pitch, box_rows)) return false;
  cache[next] = e;
  next = (next + 1) % 8;
  *out = e.map;
  return true;
}

extern cudaEvent_t g_score_ev_before, g_score_ev_after;
extern int g_score_grid;
extern int g_score_path;

// Tensor-core scoring with the finish and the selection fused in. Returns
// PQI_ENOTSUP when the device or driver lacks the feature, so the caller can
// use the CUDA-core path.
pqi_status score_tc(const pqi_weights* w, const uint32_t* theta, int shots, int spin,
                    const SelGeom& geo, float* energies, float* best_energy, int* best_index,
                    Workspace& ws, cudaStream_t s) {
  static int arch_ok = -1;
  static int num_sms = 148;
  if (arch_ok < 0) {
    int dev = 0, major = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
    arch_ok = (major == 10) ? 1 : 0;
  }
  if (!arch_ok || !encode_fn()) return PQI_ENOTSUP;
  const int n = w->n, n32 = (n + 31) >> 5, ld = w->ld;
  // int8 tensor-core operands: integer weights (one plane), or float weights
  // as four fixed-point digit planes (exact integer sums, scaled by wscale);
  // path 4 scores float weights as split bf16 instead
  const bool digits = w->kind != PQI_W_I8 && w->W_d && g_score_path != 4;
  const bool i8 = w->kind == PQI_W_I8 || digits;
  const int planes = digits ? 4 : 1;
  const double qscale = digits ? w->wscale : 1.0;
  // the int8 epilogue sums 256 columns of |Y| <= 127 n in 32 bits
  if (i8 && n > 65536) return PQI_ENOTSUP;
  const int ntn = (n + tc::BN - 1) / tc::BN;
  const int ntm = (shots + tc::BM - 1) / tc::BM;
  // 0 (default), 3 and 4: CTA pairs (cta_group::2) for more than 128
  // candidates, the A operand expanded by a separate pass and loaded by TMA;
  // 2: single CTAs, A as in 0; 5: single CTAs that expand the packed
  // candidates into the A tiles themselves
  const bool fused = g_score_path == 5;
  const bool pair = g_score_path != 2 && !fused && ntm >= 2;
  // one zeroed control block: err, mdone, key, then mcount[ntm]
  const size_t ctl_bytes = 64 + (size_t)ntm * sizeof(unsigned);
  uint8_t* ctl = ws.take<uint8_t>(ctl_bytes);
  double* qpart = ws.take<double>((size_t)ntn * shots);
  void* X = nullptr;
  if (!fused)
    X = i8 ? (void*)ws.take<int8_t>((size_t)shots * ld) : (void*)ws.take<uint16_t>((size_t)shots * ld);
  if (!ctl || !qpart || (!fused && !X)) return PQI_EINVAL;
  int* err = reinterpret_cast<int*>(ctl);
  unsigned* mdone = reinterpret_cast<unsigned*>(ctl + 8);
  unsigned long long* key = reinterpret_cast<unsigned long long*>(ctl + 16);
  unsigned* mcount = reinterpret_cast<unsigned*>(ctl + 64);
  if (i8) {
    if (!digits && !w->W_i8) return PQI_EINVAL;
  } else if (!w->W_hi || !w->W_lo) {
    return PQI_EINVAL;
  }
  const int brows = pair ? tc::BN / 2 : tc::BN;
  // the B operand's maps: int8 weights (all the same), digit planes 0..3
  // (n*ld bytes apart), or bf16 hi and lo
  const size_t plane_bytes = (size_t)n * ld;
  const void* b0 = digits ? (const void*)w->W_d : (i8 ? (const void*)w->W_i8 : (const void*)w->W_hi);
  const void* b1 = digits ? (const void*)(w->W_d + plane_bytes) : (i8 ? b0 : (const void*)w->W_lo);
  const void* b2 = digits ? (const void*)(w->W_d + 2 * plane_bytes) : b1;
  const void* b3 = digits ? (const void*)(w->W_d + 3 * plane_bytes) : b2;
  CUtensorMap ma, mb0, mb1, mb2, mb3;
  if (!cached_map(&mb0, b0, i8, n, n, ld, brows)) return PQI_ENOTSUP;
  if (!cached_map(&mb1, b1, i8, n, n, ld, brows)) return PQI_ENOTSUP;
  if (!cached_map(&mb2, b2, i8, n, n, ld, brows)) return PQI_ENOTSUP;
  if (!cached_map(&mb3, b3, i8, n, n, ld, brows)) return PQI_ENOTSUP;
  if (fused) {
    ma = mb0;  // not read: the kernel writes its A tiles itself
  } else if (!cached_map(&ma, X, i8, shots, n, ld, tc::BM)) {
    return PQI_ENOTSUP;
  }
  // kernel instances: [int8][form], form 0 = fused, 1 = single CTA, 2 = pair
  const int form = fused ? 0 : (pair ? 2 : 1);
  static const void* const kfn[2][3] = {
      {(const void*)tc::score_tc_kernel<false, false, true>, (const void*)tc::score_tc_kernel<false, false, false>,
       (const void*)tc::score_tc_kernel<false, true, false>},
      {(const void*)tc::score_tc_kernel<true, false, true>, (const void*)tc::score_tc_kernel<true, false, false>,
       (const void*)tc::score_tc_kernel<true, true, false>}};
  const int smem_bytes = fused ? tc::SMEM_BYTES_FUSED : tc::SMEM_BYTES;
  static bool attr_set[2][3] = {};
  if (!attr_set[i8][form]) {
    PQI_TRY(cudaFuncSetAttribute(kfn[i8][form], cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes));
    attr_set[i8][form] = true;
  }
  PQI_TRY(cudaMemsetAsync(ctl, 0, ctl_bytes, s));
  if (!fused) {
    const long long words = (long long)shots * n32;
    const int eg = (int)std::max<long long>(1, std::min<long long>((words + 255) / 256, 148 * 16));
    if (i8) {
      tc::expand_pm1_kernel<int8_t><<<eg, 256, 0, s>>>(theta, shots, n32, ld, (int8_t*)X);
    } else {
      tc::expand_pm1_kernel<uint16_t><<<eg, 256, 0, s>>>(theta, shots, n32, ld, (uint16_t*)X);
    }
    PQI_LAUNCHED("expand_pm1_kernel");
  }
  const int limit = g_score_grid > 0 ? g_score_grid : num_sms;
  if (g_score_ev_before) PQI_TRY(cudaEventRecord(g_score_ev_before, s));
  if (pair) {
    const int tiles = ntn * ((shots + 2 * tc::BM - 1) / (2 * tc::BM));
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(tc::PTHREADS);
    cfg.dynamicSmemBytes = tc::SMEM_BYTES;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // a persistent grid of exactly the pairs that can be resident at once (a
    // pair needs two free SMs of one GPC), cached per weight kind
    static int fit[2] = {0, 0};
    if (!fit[i8]) {
      cfg.gridDim = dim3(2);
      int f = 0;
      PQI_TRY(cudaOccupancyMaxActiveClusters(&f, kfn[i8][2], &cfg));
      fit[i8] = std::max(1, f);
    }
    const int pairs = std::max(1, std::min({tiles, limit / 2, fit[i8]}));
    cfg.gridDim = dim3(2 * pairs);
    if (i8) {
      PQI_TRY(cudaLaunchKernelEx(&cfg, tc::score_tc_kernel<true, true, false>, ma, mb0, mb1, mb2, mb3, planes, qscale, n, shots,
                                 theta, n32, w->upper_sum, spin, geo, qpart, energies, mcount,
                                 mdone, key, best_energy, best_index, err));
    } else {
      PQI_TRY(cudaLaunchKernelEx(&cfg, tc::score_tc_kernel<false, true, false>, ma, mb0, mb1, mb2, mb3, planes, qscale, n, shots,
                                 theta, n32, w->upper_sum, spin, geo, qpart, energies, mcount,
                                 mdone, key, best_energy, best_index, err));
    }
  } else {
    const int grid = std::min(ntn * ntm, limit);
    const int threads = fused ? tc::FTHREADS : tc::PTHREADS;
    if (i8) {
      auto k = fused ? tc::score_tc_kernel<true, false, true> : tc::score_tc_kernel<true, false, false>;
      k<<<grid, threads, smem_bytes, s>>>(ma, mb0, mb1, mb2, mb3, planes, qscale, n, shots, theta, n32, w->upper_sum, spin, geo,
                                          qpart, energies, mcount, mdone, key, best_energy, best_index,
                                          err);
    } else {
      auto k = fused ? tc::score_tc_kernel<false, false, true> : tc::score_tc_kernel<false, false, false>;
      k<<<grid, threads, smem_bytes, s>>>(ma, mb0, mb1, mb2, mb3, planes, qscale, n, shots, theta, n32, w->upper_sum, spin, geo,
                                          qpart, energies, mcount, mdone, key, best_energy, best_index,
                                          err);
    }
  }
  PQI_LAUNCHED("score_tc_kernel");
  if (g_score_ev_after) PQI_TRY(cudaEventRecord(g_score_ev_after, s));
  return PQI_OK;
}

}  // namespace pqi
