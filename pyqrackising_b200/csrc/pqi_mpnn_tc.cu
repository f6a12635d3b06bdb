// libpqi: tensor-core (tcgen05) message products of the learned proposal
// network: OUT[:, 0:64] = A_hat X for the dense normalised adjacency A_hat
// (n x n bf16, symmetric, so the same product serves the forward messages and
// the backward message gradients) and a 64-column activation X, given as its
// transpose Xt (64 x n, K-major like A_hat's rows).
//
// One CTA per 128-row tile of the output, K = n walked in 64-element stages
// through a 4-stage TMA ring; kind::f16 MMAs (bf16 A and B, M = 128, N = 64,
// K = 16) accumulate in 64 TMEM columns (float32); four epilogue warps read
// their lane quarter and write bf16 and / or float32 (optionally adding the
// float32 output already there). Warp 0 issues TMA, warp 1 owns TMEM and
// issues the MMAs. Every mbarrier wait is bounded; on expiry the tile's
// outputs are NaN (the caller's finiteness check then takes the fallback) and
// TMEM is still released.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>

#include "pqi_common.cuh"
#include "pqi_tc.cuh"

namespace pqi {

namespace mtc {

constexpr int TM = 128;                       // output rows per CTA
constexpr int TN = 64;                        // output columns (hidden width)
constexpr int TKE = 64;                       // K elements per stage (128 bytes of bf16)
constexpr int STAGES = 4;
constexpr int A_STAGE = TM * 128;             // 16 KB
constexpr int B_STAGE = TN * 128;             // 8 KB
constexpr int STAGE_BYTES = A_STAGE + B_STAGE;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;
constexpr int THREADS = 192;
constexpr uint32_t kIdesc = (1u << 4)     // D: f32
                            | (1u << 7)   // A: bf16
                            | (1u << 10)  // B: bf16
                            | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);

__global__ void __launch_bounds__(THREADS, 1)
    adj_gemm_kernel(const __grid_constant__ CUtensorMap map_a,
                    const __grid_constant__ CUtensorMap map_b, int n, float beta,
                    float* __restrict__ out32, __nv_bfloat16* __restrict__ out16, int ldo) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[STAGES];
  __shared__ __align__(8) uint64_t empty_bar[STAGES];
  __shared__ __align__(8) uint64_t acc_bar;
  __shared__ uint32_t tmem_holder;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t raw = tc::smem_u32(smem_raw);
  uint8_t* smem = smem_raw + ((1024 - (raw & 1023)) & 1023);
  const int m0 = blockIdx.x * TM;
  const int kblocks = (n + TKE - 1) / TKE;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(&full_bar[s], 1);
      tc::mbar_init(&empty_bar[s], 1);
    }
    tc::mbar_init(&acc_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32(&tmem_holder)),
                 "r"(TN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_holder;

  if (warp == 0) {
    if (lane == 0) {
      for (int kb = 0; kb < kblocks; ++kb) {
        const int s = kb % STAGES;
        // (a wait that runs out stops the loads; the epilogue then writes NaN)
        if (kb >= STAGES && !tc::mbar_wait(&empty_bar[s], ((kb / STAGES) - 1) & 1)) break;
        uint8_t* dst = smem + s * STAGE_BYTES;
        tc::mbar_expect_tx(&full_bar[s], STAGE_BYTES);
        tc::tma_load_2d(dst, &map_a, &full_bar[s], kb * TKE, m0);
        tc::tma_load_2d(dst + A_STAGE, &map_b, &full_bar[s], kb * TKE, 0);
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      bool ok = true;
      for (int kb = 0; kb < kblocks; ++kb) {
        const int s = kb % STAGES;
        if (!tc::mbar_wait(&full_bar[s], (kb / STAGES) & 1)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a_addr = tc::smem_u32(smem + s * STAGE_BYTES);
        const uint32_t b_addr = a_addr + A_STAGE;
#pragma unroll
        for (int k = 0; k < 4; ++k)  // K = 16 bf16 = 32 bytes per MMA
          tc::mma<false>(tmem, tc::sw128_desc(a_addr + k * 32), tc::sw128_desc(b_addr + k * 32),
                         kIdesc, (kb > 0 || k > 0) ? 1u : 0u);
        tc::mma_commit(&empty_bar[s]);
      }
      if (ok) tc::mma_commit(&acc_bar);
    }
    __syncwarp();
  } else {
    // epilogue: warp w reads TMEM lanes 32 * (w % 4) .. + 31 = output rows
    const int quarter = warp & 3;
    const int row = m0 + quarter * 32 + lane;
    const bool ready = tc::mbar_wait(&acc_bar, 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    uint32_t r[64];
    if (__all_sync(0xFFFFFFFFu, ready)) {
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16);
      tc::tmem_load32_nowait(taddr, *reinterpret_cast<uint32_t(*)[32]>(&r[0]));
      tc::tmem_load32_nowait(taddr + 32, *reinterpret_cast<uint32_t(*)[32]>(&r[32]));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      tc::reg_fence32(*reinterpret_cast<uint32_t(*)[32]>(&r[0]));
      tc::reg_fence32(*reinterpret_cast<uint32_t(*)[32]>(&r[32]));
    } else {
#pragma unroll
      for (int c = 0; c < 64; ++c) r[c] = 0x7FC00000u;  // NaN
    }
    if (row < n) {
      float* o32 = out32 ? out32 + (size_t)row * ldo : nullptr;
      __nv_bfloat16* o16 = out16 ? out16 + (size_t)row * ldo : nullptr;
#pragma unroll
      for (int c = 0; c < 64; c += 2) {
        float v0 = __uint_as_float(r[c]), v1 = __uint_as_float(r[c + 1]);
        if (o32) {
          if (beta != 0.0f) {
            v0 += beta * o32[c];
            v1 += beta * o32[c + 1];
          }
          o32[c] = v0;
          o32[c + 1] = v1;
        }
        if (o16) *reinterpret_cast<__nv_bfloat162*>(o16 + c) = __floats2bfloat162_rn(v0, v1);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN));
}

// Xt[c][r] = X[r][c] for r < n, c < 64 (bf16; X row pitch ldx, Xt row pitch ldt)
__global__ void transpose64_kernel(const __nv_bfloat16* __restrict__ X, int n, int ldx,
                                   __nv_bfloat16* __restrict__ Xt, int ldt) {
  __shared__ __nv_bfloat16 tile[64][65];
  const int r0 = blockIdx.x * 64;
  for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
    const int rr = e >> 6, c = e & 63;
    tile[rr][c] = (r0 + rr < n) ? X[(size_t)(r0 + rr) * ldx + c] : __float2bfloat16_rn(0.0f);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
    const int c = e >> 6, rr = e & 63;
    if (r0 + rr < ldt) Xt[(size_t)c * ldt + r0 + rr] = tile[rr][c];
  }
}

}  // namespace mtc

}  // namespace pqi

using namespace pqi;

extern "C" {

pqi_status pqi_mpnn_transpose64(const void* X, int n, int ldx, void* Xt, int ldt, void* stream) {
  PQI_CHECK_ARG(X && Xt && n > 0 && ldx >= 64 && ldt >= n);
  mtc::transpose64_kernel<<<(std::max(n, ldt) + 63) / 64, 256, 0, as_stream(stream)>>>(
      static_cast<const __nv_bfloat16*>(X), n, ldx, static_cast<__nv_bfloat16*>(Xt), ldt);
  PQI_LAUNCHED("transpose64_kernel");
  return PQI_OK;
}

pqi_status pqi_mpnn_adj_gemm(const void* Ahat, int ld, int n, const void* Xt, int ldt, float beta,
                             float* out32, void* out16, int ldo, void* stream) {
  PQI_CHECK_ARG(Ahat && Xt && (out32 || out16) && n > 0 && ldo >= 64);
  PQI_CHECK_ARG(beta == 0.0f || out32);
  // TMA: 16-byte aligned bases and row pitches
  PQI_CHECK_ARG(ld >= n && ld % 8 == 0 && ldt >= n && ldt % 8 == 0);
  PQI_CHECK_ARG(((uintptr_t)Ahat & 15) == 0 && ((uintptr_t)Xt & 15) == 0);
  PQI_CHECK_ARG(ldo % 2 == 0 && (!out16 || ((uintptr_t)out16 & 3) == 0));
  int dev = 0, major = 0;
  PQI_TRY(cudaGetDevice(&dev));
  PQI_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  if (major != 10 || !encode_fn()) return PQI_ENOTSUP;
  CUtensorMap ma, mb;
  if (!cached_map(&ma, Ahat, false, n, n, ld, mtc::TM)) return PQI_ENOTSUP;
  if (!cached_map(&mb, Xt, false, mtc::TN, n, ldt, mtc::TN)) return PQI_ENOTSUP;
  static bool attr = false;
  if (!attr) {
    PQI_TRY(cudaFuncSetAttribute(mtc::adj_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 mtc::SMEM_BYTES));
    attr = true;
  }
  mtc::adj_gemm_kernel<<<(n + mtc::TM - 1) / mtc::TM, mtc::THREADS, mtc::SMEM_BYTES,
                         as_stream(stream)>>>(ma, mb, n, beta, out32,
                                              static_cast<__nv_bfloat16*>(out16), ldo);
  PQI_LAUNCHED("adj_gemm_kernel");
  return PQI_OK;
}

}  // extern "C"
