// libpqi: the TFIM-inspired candidate sampler of maxcut_tfim on the GPU
// (pyqrackising/maxcut_tfim.py:36-74, 139-145, 189-209 and
// maxcut_tfim_util.py:545-724).
//
//  * tfim_jz: per-node mean coupling J_eff and degree (init_J_and_z).
//  * tfim_cdf: the Hamming-weight distribution (maxcut_hamming_cdf with
//    probability_by_hamming_weight and _apply_time_envelope), float64, in two
//    passes: per (step, node) pair the two normalisers, then per bin the sum
//    over pairs in a fixed order.
//  * tfim_sample: one warp per shot draws a Hamming weight from the CDF
//    (sample_mag) and picks nodes with multiplicative repulsion
//    (local_repulsion_choice, bit_pick), float64 weights so a weight that
//    underflows to zero counts as picked exactly as in the reference. The
//    selection mask is written as packed bits for the scoring kernel.
// Random numbers: a counter-based generator keyed by (seed, round, shot,
// draw), so a run is reproducible for a given seed (the reference's numba
// generator is unseeded and not reproducible, maxcut_tfim_util.py:692,715).
#include <algorithm>

#include "pqi_common.cuh"

namespace pqi {

constexpr double kEps = 1.1920928955078125e-07;  // float32 epsilon, the reference's `epsilon`
constexpr double kPi = 3.141592653589793;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  // SplitMix64 finaliser (Steele, Lea, Flood 2014)
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// uniform double in [0, 1) from a counter
__device__ __forceinline__ double uniform(uint64_t seed, uint64_t round, uint64_t shot,
                                          uint64_t draw) {
  uint64_t h = mix64(seed ^ mix64(round * 0x632BE59BD9B4E019ull + shot));
  h = mix64(h ^ (draw * 0xD1B54A32D192ED03ull));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

// ---------------------------------------------------------------------------
// init_J_and_z (maxcut_tfim.py:189-209): G_min over all of W (diagonal
// included); per row, entries with W - G_min > eps count as edges.

__global__ void tfim_min_kernel(const float* __restrict__ W, long long total, float* out_min) {
  __shared__ float red[32];
  float m = INFINITY;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x)
    m = fminf(m, W[e]);
  for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : INFINITY;
    for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    if (threadIdx.x == 0) {
      // order-preserving for floats of either sign: store as int via ordered key
      unsigned int k = __float_as_uint(m);
      k = (k & 0x80000000u) ? ~k : (k | 0x80000000u);
      atomicMin(reinterpret_cast<unsigned int*>(out_min), k);
    }
  }
}

__global__ void tfim_jz_kernel(const float* __restrict__ W, int n, const float* min_key,
                               double* __restrict__ J_eff, unsigned int* __restrict__ degrees) {
  unsigned int k = *reinterpret_cast<const unsigned int*>(min_key);
  k = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
  const float gmin = __uint_as_float(k);
  const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  for (int r = blockIdx.x * warps + (threadIdx.x >> 5); r < n; r += gridDim.x * warps) {
    const float* row = W + (size_t)r * n;
    unsigned int deg = 0;
    double J = 0.0;
    for (int m = lane; m < n; m += 32) {
      const float val = row[m] - gmin;  // float32, as the reference
      if ((double)val <= kEps) continue;
      ++deg;
      J += (double)val;
    }
    for (int o = 16; o > 0; o >>= 1) {
      deg += __shfl_xor_sync(0xFFFFFFFFu, deg, o);
      J += __shfl_xor_sync(0xFFFFFFFFu, J, o);
    }
    if (lane == 0) {
      J_eff[r] = deg > 0 ? -J / (double)deg : 0.0;
      degrees[r] = deg;
    }
  }
}

// The sparse path's J_eff and degrees (maxcut_tfim_sparse.py:204-224): the
// same rule, but the reference runs it as plain numpy scalar arithmetic, so
// the row sum is float32, accumulated in node order, and J = -(sum / degree)
// is a float32 division. One thread per row reproduces that order exactly.
__global__ void tfim_jz_f32_kernel(const float* __restrict__ W, int n, const float* min_key,
                                   double* __restrict__ J_eff, unsigned int* __restrict__ degrees) {
  unsigned int k = *reinterpret_cast<const unsigned int*>(min_key);
  k = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
  const float gmin = __uint_as_float(k);
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const float* row = W + (size_t)r * n;
    unsigned int deg = 0;
    float J = 0.0f;
    for (int m = 0; m < n; ++m) {
      const float val = __fsub_rn(row[m], gmin);
      if ((double)val <= kEps) continue;
      ++deg;
      J = __fadd_rn(J, val);
    }
    J_eff[r] = deg > 0 ? (double)(-__fdiv_rn(J, (float)deg)) : 0.0;
    degrees[r] = deg;
  }
}

// ---------------------------------------------------------------------------
// maxcut_hamming_cdf (maxcut_tfim_util.py:654-687)

struct CdfParams {
  int n;           // nodes; bins are 0..n
  int n_steps;     // 1 << quality
  double delta_t;  // tot_t / n_steps
  double tot_t;
  double h_mult;   // |anneal_h|
  double omega;
};

// p of probability_by_hamming_weight (util:627-631) for node q at time t
__device__ __forceinline__ double pbhw_p(double J, double h, double z, double theta, double t,
                                         double omega) {
  const double zJ = z * J;
  const double theta_c =
      fabs(zJ) < kEps ? ((J > 0 ? kPi : -kPi) / 2) : asin(fmax(-1.0, fmin(1.0, h / zJ)));
  return exp2(fabs(J / h) - 1.0) *
             (1.0 + sin(theta - theta_c) * cos(omega * J * t + theta) / (1.0 + sqrt(t))) -
         0.5;
}

// unnormalised envelope term of bin k: factor^(k+1) * exp(-|k - n/2| / t_eff)
__device__ __forceinline__ double env_term(double log2f, int k, double half, double t_eff,
                                           double* bias_out) {
  const double b = exp2(log2f * (double)(k + 1));
  if (bias_out) *bias_out = b;
  return b * exp(-fabs((double)k - half) / t_eff);
}

// Pass 1: one block per (step, node) pair (grid-stride). For both t and t - dt
// store S = sum_k bias_k and E = sum_k (bias_k / S) env_k, or -1 when J_eff is
// skipped (|J| < eps). J_eff = -(mean positive excess) <= 0, so the reversed,
// unnormalised J > 0 branch of probability_by_hamming_weight never applies.
__global__ void tfim_cdf_norms_kernel(CdfParams P, const double* __restrict__ J_eff,
                                      const unsigned int* __restrict__ degrees,
                                      double* __restrict__ norms, double* __restrict__ pvals) {
  __shared__ double red[2][32];
  const int n = P.n, n_bias = n + 1;
  const double half = n / 2.0;
  const long long pairs = (long long)(P.n_steps - 1) * n;
  for (long long pr = blockIdx.x; pr < pairs; pr += gridDim.x) {
    const int step = 1 + (int)(pr / n), q = (int)(pr % n);
    const double J = J_eff[q];
    double* nm = norms + pr * 4;
    if (fabs(J) < kEps) {
      if (threadIdx.x == 0) nm[0] = -1.0;
      continue;
    }
    const double z = (double)degrees[q];
    const double zJ0 = z * J;
    const double theta =
        fabs(zJ0) < kEps ? ((J > 0 ? kPi : -kPi) / 2) : asin(fmax(-1.0, fmin(1.0, P.h_mult / zJ0)));
    const double t = step * P.delta_t, tm1 = (step - 1) * P.delta_t;
    const double h_t = P.h_mult * (P.tot_t - t);
    for (int which = 0; which < 2; ++which) {
      const double tt = which == 0 ? t : tm1;
      const double p = pbhw_p(J, h_t, z, theta, tt, P.omega);
      const double log2f = -p / n_bias;
      const double t_eff = tt > 1e-9 ? tt : 1e-9;
      double sb = 0.0, se = 0.0;
      for (int k = threadIdx.x; k < n_bias; k += blockDim.x) {
        double b;
        se += env_term(log2f, k, half, t_eff, &b);
        sb += b;
      }
      for (int o = 16; o > 0; o >>= 1) {
        sb += __shfl_xor_sync(0xFFFFFFFFu, sb, o);
        se += __shfl_xor_sync(0xFFFFFFFFu, se, o);
      }
      const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
      if (lane == 0) {
        red[0][w] = sb;
        red[1][w] = se;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double SB = 0.0, SE = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
          SB += red[0][i];
          SE += red[1][i];
        }
        nm[2 * which] = SB;
        nm[2 * which + 1] = SE / SB;  // sum of the envelope over bias / S
        pvals[pr * 2 + which] = log2f;
      }
      __syncthreads();
    }
  }
}

// Pass 2: thread per bin k, over all pairs in order: hamming_prob[k] +=
// envelope(t)[k] - envelope(t - dt)[k], each normalised (util:675-676).
__global__ void tfim_cdf_accum_kernel(CdfParams P, const double* __restrict__ J_eff,
                                      const double* __restrict__ norms,
                                      const double* __restrict__ pvals,
                                      double* __restrict__ hprob) {
  const int n = P.n, n_bias = n + 1;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_bias) return;
  const double half = n / 2.0;
  const int mid = n / 2;
  double acc = hprob[k];
  const long long pairs = (long long)(P.n_steps - 1) * n;
  for (long long pr = 0; pr < pairs; ++pr) {
    const double* nm = norms + pr * 4;
    if (nm[0] < 0.0) continue;
    const int step = 1 + (int)(pr / n);
    double v[2];
    for (int which = 0; which < 2; ++which) {
      const double tt = which == 0 ? step * P.delta_t : (step - 1) * P.delta_t;
      const double t_eff = tt > 1e-9 ? tt : 1e-9;
      const double S = nm[2 * which], E = nm[2 * which + 1];
      if (!(E > 0.0)) {
        v[which] = (k == mid) ? 1.0 : 0.0;  // underflow: delta at half filling (util:612-618)
      } else {
        v[which] = env_term(pvals[pr * 2 + which], k, half, t_eff, nullptr) / S / E;
      }
    }
    acc += v[0] - v[1];
  }
  hprob[k] = acc;
}

// normalise and accumulate the CDF over bins 1..n-1 (util:678-687); one block.
__global__ void tfim_cdf_finish_kernel(int n, const double* __restrict__ hprob,
                                       double* __restrict__ cum) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int k = 0; k <= n; ++k) s += hprob[k];
  const double denom = s - (hprob[0] + hprob[n]);
  double tot = 0.0;
  for (int i = 0; i < n - 1; ++i) {
    tot += hprob[i + 1] / denom;
    cum[i] = tot;
  }
  cum[n - 2] = 1.0;
}

// ---------------------------------------------------------------------------
// Sampler: one warp per shot; lane l owns nodes [l*C, (l+1)*C), C = ceil(n/32).

// sample_mag (util:691-707), step for step: bisect for an m with cum[m] >= p
// and (m == 0 or cum[m-1] < p). The reference's cumulative array need not be
// monotone (it accumulates differences of distributions), so this is not a
// plain lower bound; the same probes give the same m. The loop is capped at 64
// probes (the reference loops until the condition holds).
__device__ __forceinline__ int sample_mag(const double* cum, int len, double p) {
  int left = 0, right = len - 1, m = 0;
  for (int it = 0; it < 64; ++it) {
    m = (left + right) >> 1;
    if (cum[m] >= p && (m == 0 || cum[m - 1] < p)) break;
    if (cum[m] < p) {
      left = m + 1;
    } else {
      right = m - 1;
    }
  }
  return m;
}

constexpr int kWtsPitch = 33;  // doubles per row of a warp's weight table (32 lanes + 1)
constexpr int kRowBatch = 16;  // row steps of 32 weights in flight per repulsion update

// base^(-w) for a weight other than +-1, out of line: the unrolled update loop
// stays small enough for the instruction cache
__device__ __noinline__ double repulsion_factor(double lnb, float wv) {
  return exp(-lnb * (double)wv);
}

// adj_ptr / adj_col / adj_val (nullable): the nonzero entries of each row of W
// in column order; when given, a repulsion update walks the picked node's
// list instead of scanning its dense row (the same multiplications).
__global__ void tfim_sample_kernel(const float* __restrict__ W, int n,
                                   const double* __restrict__ cum, int ncum, double base,
                                   int repel, uint64_t seed, uint64_t round, int shots,
                                   uint32_t* __restrict__ theta_out, double* __restrict__ wglob,
                                   int use_smem, const long long* __restrict__ adj_ptr,
                                   const int* __restrict__ adj_col,
                                   const float* __restrict__ adj_val) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  const int C = (n + 31) >> 5;
  const int n32 = C;  // words per packed row == nodes per lane chunk, both ceil(n/32)
  double* wts = use_smem ? reinterpret_cast<double*>(smem) + (size_t)wib * (C * kWtsPitch)
                         : wglob + (size_t)(blockIdx.x * wpb + wib) * (C * kWtsPitch);
  const double lnb = log(base);
  const double rep1 = exp(-lnb);  // repulsion factors of the weights +1 and -1
  const double repm1 = exp(lnb);
  for (int s = blockIdx.x * wpb + wib; s < shots; s += gridDim.x * wpb) {
    const int m = sample_mag(cum, ncum, uniform(seed, round, (uint64_t)s, 0));
    const int node0 = s % n;
    uint32_t* out = theta_out + (size_t)s * n32;
    if (m == 1) {
      for (int w = lane; w < n32; w += 32) out[w] = (w == (node0 >> 5)) ? (1u << (node0 & 31)) : 0u;
      continue;
    }
    // lane l owns nodes v0 .. v0 + C - 1 (the bisection's order); node v0 + i
    // is stored at wts[i * 33 + l]: the owners' sweeps (fixed i, 32 lanes) and
    // the node-order sweeps (32 consecutive nodes) both spread over the banks
    const int v0 = lane * C;
    for (int i = 0; i < C; ++i) wts[i * kWtsPitch + lane] = (v0 + i < n) ? 1.0 : 0.0;
    __syncwarp();
    // picks after the first node: m - 1 for m >= 2, one for m == 0 (the loop of
    // local_repulsion_choice runs max(0, m - 2) times, then one last pick)
    const int picks = (m == 0) ? 1 : m - 1;
    int node = node0;
    for (int j = 0; j <= picks; ++j) {
      if (j > 0) {
        // bit_pick (util:711-724): p = sum(weights) * u, first i with p < running sum.
        // The lane's sum runs as four interleaved partial sums (independent
        // adds instead of one chain of C).
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        int i = 0;
        for (; i + 3 < C; i += 4) {
          a0 += wts[i * kWtsPitch + lane];
          a1 += wts[(i + 1) * kWtsPitch + lane];
          a2 += wts[(i + 2) * kWtsPitch + lane];
          a3 += wts[(i + 3) * kWtsPitch + lane];
        }
        for (; i < C; ++i) a0 += wts[i * kWtsPitch + lane];
        const double loc = (a0 + a1) + (a2 + a3);
        double incl = loc;
        for (int o = 1; o < 32; o <<= 1) {
          const double y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
          if (lane >= o) incl += y;
        }
        const double total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        const double p = total * uniform(seed, round, (uint64_t)s, (uint64_t)j);
        const unsigned hit = __ballot_sync(0xFFFFFFFFu, p < incl);
        int picked = 0;
        if (hit) {
          // lane l's chunk holds the pick: the whole warp scans its C weights,
          // 32 at a time (inclusive warp scan on top of the running sum)
          const int l = __ffs(hit) - 1;
          double run = __shfl_sync(0xFFFFFFFFu, incl - loc, l);
          picked = l * C;  // no prefix above p (rounding): the chunk's first node
          for (int i0 = 0; i0 < C; i0 += 32) {
            const int ii = i0 + lane;
            double w = (ii < C) ? wts[ii * kWtsPitch + l] : 0.0;
            for (int o = 1; o < 32; o <<= 1) {
              const double y = __shfl_up_sync(0xFFFFFFFFu, w, o);
              if (lane >= o) w += y;
            }
            const unsigned h2 = __ballot_sync(0xFFFFFFFFu, ii < C && p < run + w);
            if (h2) {
              picked = l * C + i0 + __ffs(h2) - 1;
              break;
            }
            run += __shfl_sync(0xFFFFFFFFu, w, 31);
          }
        }
        node = picked;
      }
      // update_repulsion_choice (maxcut_tfim.py:37-45) for all but the last pick
      __syncwarp();
      if (lane == (node / C)) wts[(node - lane * C) * kWtsPitch + lane] = 0.0;
      __syncwarp();
      if (j < picks && repel && adj_ptr) {
        // the picked node's nonzero weights, 32 list entries per step
        const long long e1 = adj_ptr[node + 1];
        for (long long e = adj_ptr[node] + lane; e < e1; e += 32) {
          const int v = adj_col[e];
          const float wv = adj_val[e];
          const int q = v / C;
          wts[(v - q * C) * kWtsPitch + q] *= (wv == 1.0f)    ? rep1
                                              : (wv == -1.0f) ? repm1
                                                              : repulsion_factor(lnb, wv);
        }
      } else if (j < picks && repel) {
        // the row in node order, 32 consecutive weights per step (coalesced),
        // kRowBatch steps loaded before any is applied (the weight table may
        // be global memory, so loads would otherwise wait behind the stores);
        // each lane scales the weight of its node v wherever v's owner keeps it
        const float* row = W + (size_t)node * n;
        int q = lane / C, r = lane - q * C;  // v = lane + 32 w = q C + r
        const int dq = 32 / C, dr = 32 - dq * C;
        for (int vb = lane; vb < n; vb += 32 * kRowBatch) {
          float wv[kRowBatch];
#pragma unroll
          for (int u = 0; u < kRowBatch; ++u) wv[u] = (vb + 32 * u < n) ? __ldg(row + vb + 32 * u) : 0.0f;
#pragma unroll
          for (int u = 0; u < kRowBatch; ++u) {
            if (wv[u] != 0.0f)
              wts[r * kWtsPitch + q] *= (wv[u] == 1.0f)    ? rep1
                                        : (wv[u] == -1.0f) ? repm1
                                                           : repulsion_factor(lnb, wv[u]);
            q += dq;
            r += dr;
            if (r >= C) {
              r -= C;
              ++q;
            }
          }
        }
      }
      __syncwarp();
    }
    // selection mask: weights == 0 (picked, or underflowed to zero)
    for (int w = 0; w < n32; ++w) {
      const int v = w * 32 + lane;
      const bool sel = v < n && wts[(v % C) * kWtsPitch + v / C] == 0.0;
      const unsigned bits = __ballot_sync(0xFFFFFFFFu, sel);
      if (lane == 0) out[w] = bits;
    }
    __syncwarp();
  }
}

// Nonzero counts of W's rows (warp per row).
__global__ void tfim_adj_count_kernel(const float* __restrict__ W, int n, long long* __restrict__ count) {
  const int lane = threadIdx.x & 31;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += (gridDim.x * blockDim.x) >> 5) {
    const float* row = W + (size_t)r * n;
    int c = 0;
    for (int v0 = 0; v0 < n; v0 += 32) {
      const int v = v0 + lane;
      c += __popc(__ballot_sync(0xFFFFFFFFu, v < n && row[v] != 0.0f));
    }
    if (lane == 0) count[r] = c;
  }
}

// Row lists in column order at adj_ptr[r] (warp per row, ballot compaction).
__global__ void tfim_adj_fill_kernel(const float* __restrict__ W, int n,
                                     const long long* __restrict__ adj_ptr, int* __restrict__ adj_col,
                                     float* __restrict__ adj_val) {
  const int lane = threadIdx.x & 31;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += (gridDim.x * blockDim.x) >> 5) {
    const float* row = W + (size_t)r * n;
    long long at = adj_ptr[r];
    for (int v0 = 0; v0 < n; v0 += 32) {
      const int v = v0 + lane;
      const float w = v < n ? row[v] : 0.0f;
      const unsigned nz = __ballot_sync(0xFFFFFFFFu, w != 0.0f);
      if (w != 0.0f) {
        const long long e = at + __popc(nz & ((1u << lane) - 1u));
        adj_col[e] = v;
        adj_val[e] = w;
      }
      at += __popc(nz);
    }
  }
}

}  // namespace pqi

using namespace pqi;

extern "C" {

pqi_status pqi_tfim_jz(const float* W, int n, double* J_eff, unsigned int* degrees,
                       void* workspace, size_t workspace_bytes, void* stream) {
  PQI_CHECK_ARG(W && J_eff && degrees && n > 0);
  Workspace ws(workspace, workspace_bytes);
  float* mn = ws.take<float>(1);
  PQI_CHECK_ARG(mn);
  cudaStream_t s = as_stream(stream);
  PQI_TRY(cudaMemsetAsync(mn, 0xFF, sizeof(float), s));  // max key
  const long long total = (long long)n * n;
  const int g = (int)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148 * 8));
  tfim_min_kernel<<<g, 256, 0, s>>>(W, total, mn);
  PQI_LAUNCHED("tfim_min_kernel");
  tfim_jz_kernel<<<std::max(1, std::min((n + 7) / 8, 148 * 4)), 256, 0, s>>>(W, n, mn, J_eff,
                                                                             degrees);
  PQI_LAUNCHED("tfim_jz_kernel");
  return PQI_OK;
}

pqi_status pqi_tfim_jz_f32(const float* W, int n, double* J_eff, unsigned int* degrees,
                           void* workspace, size_t workspace_bytes, void* stream) {
  PQI_CHECK_ARG(W && J_eff && degrees && n > 0);
  Workspace ws(workspace, workspace_bytes);
  float* mn = ws.take<float>(1);
  PQI_CHECK_ARG(mn);
  cudaStream_t s = as_stream(stream);
  PQI_TRY(cudaMemsetAsync(mn, 0xFF, sizeof(float), s));  // max key
  const long long total = (long long)n * n;
  const int g = (int)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148 * 8));
  tfim_min_kernel<<<g, 256, 0, s>>>(W, total, mn);
  PQI_LAUNCHED("tfim_min_kernel");
  tfim_jz_f32_kernel<<<(n + 127) / 128, 128, 0, s>>>(W, n, mn, J_eff, degrees);
  PQI_LAUNCHED("tfim_jz_f32_kernel");
  return PQI_OK;
}

size_t pqi_tfim_cdf_workspace_bytes(int n, int quality) {
  const long long pairs = (long long)((1 << quality) - 1) * n;
  return (size_t)pairs * 6 * sizeof(double) + (size_t)(n + 1) * sizeof(double) + 4096;
}

pqi_status pqi_tfim_cdf(const double* J_eff, const unsigned int* degrees, int n, int quality,
                        double anneal_t, double anneal_h, const double* thresholds, double* cum,
                        void* workspace, size_t workspace_bytes, void* stream) {
  PQI_CHECK_ARG(J_eff && degrees && thresholds && cum && n >= 3 && quality >= 0 && quality < 30);
  Workspace ws(workspace, workspace_bytes);
  const long long pairs = (long long)((1 << quality) - 1) * n;
  double* norms = ws.take<double>((size_t)std::max<long long>(pairs, 1) * 4);
  double* pvals = ws.take<double>((size_t)std::max<long long>(pairs, 1) * 2);
  double* hprob = ws.take<double>((size_t)n + 1);
  PQI_CHECK_ARG(norms && pvals && hprob);
  cudaStream_t s = as_stream(stream);
  PQI_TRY(cudaMemcpyAsync(hprob, thresholds, sizeof(double) * (n + 1), cudaMemcpyDeviceToDevice, s));
  CdfParams P;
  P.n = n;
  P.n_steps = 1 << quality;
  P.tot_t = anneal_t;
  P.delta_t = anneal_t / P.n_steps;
  P.h_mult = fabs(anneal_h);
  P.omega = 1.5 * kPi;
  if (pairs > 0) {
    const int g = (int)std::min<long long>(pairs, 148 * 16);
    tfim_cdf_norms_kernel<<<g, 256, 0, s>>>(P, J_eff, degrees, norms, pvals);
    PQI_LAUNCHED("tfim_cdf_norms_kernel");
    tfim_cdf_accum_kernel<<<(n + 1 + 127) / 128, 128, 0, s>>>(P, J_eff, norms, pvals, hprob);
    PQI_LAUNCHED("tfim_cdf_accum_kernel");
  }
  tfim_cdf_finish_kernel<<<1, 32, 0, s>>>(n, hprob, cum);
  PQI_LAUNCHED("tfim_cdf_finish_kernel");
  return PQI_OK;
}

size_t pqi_tfim_sample_workspace_bytes(int n) {
  const int C = (n + 31) / 32;
  return (size_t)148 * 16 * kWtsPitch * C * sizeof(double) + 4096;
}

static pqi_status tfim_sample_impl(const float* W, int n, const double* cum, double repulsion_base,
                                   uint64_t seed, uint64_t round, int shots, uint32_t* theta_out,
                                   void* workspace, size_t workspace_bytes, void* stream,
                                   const long long* adj_ptr, const int* adj_col, const float* adj_val) {
  // W is read only without row lists (the dense row scan)
  PQI_CHECK_ARG((W || adj_ptr) && cum && theta_out && n >= 3 && shots > 0);
  cudaStream_t s = as_stream(stream);
  const int C = (n + 31) / 32;
  const size_t per_warp = (size_t)C * kWtsPitch * sizeof(double);
  const int repel = fabs(1.0 - repulsion_base) <= kEps ? 0 : 1;
  int wpb = 4;
  size_t smem = per_warp * wpb;
  int use_smem = 1;
  double* wglob = nullptr;
  int grid;
  if (smem <= 160 * 1024) {
    grid = (int)std::min<long long>(((long long)shots + wpb - 1) / wpb, 148 * 8);
    static size_t set_bytes = 0;
    if (smem > 48 * 1024 && smem > set_bytes) {
      PQI_TRY(cudaFuncSetAttribute(tfim_sample_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
      set_bytes = smem;
    }
  } else {
    use_smem = 0;
    smem = 0;
    Workspace ws(workspace, workspace_bytes);
    const size_t avail = workspace_bytes > 8192 ? workspace_bytes - 8192 : 0;
    const long long warps = std::min<long long>((long long)(avail / per_warp), 148 * 16);
    PQI_CHECK_ARG(warps >= wpb);
    grid = (int)std::min<long long>(warps / wpb, ((long long)shots + wpb - 1) / wpb);
    wglob = ws.take<double>((size_t)grid * wpb * C * kWtsPitch);
    PQI_CHECK_ARG(wglob);
  }
  tfim_sample_kernel<<<grid, 32 * wpb, smem, s>>>(W, n, cum, n - 1, repulsion_base, repel, seed,
                                                   round, shots, theta_out, wglob, use_smem,
                                                   adj_ptr, adj_col, adj_val);
  PQI_LAUNCHED("tfim_sample_kernel");
  return PQI_OK;
}

pqi_status pqi_tfim_sample(const float* W, int n, const double* cum, double repulsion_base,
                           uint64_t seed, uint64_t round, int shots, uint32_t* theta_out,
                           void* workspace, size_t workspace_bytes, void* stream) {
  return tfim_sample_impl(W, n, cum, repulsion_base, seed, round, shots, theta_out, workspace,
                          workspace_bytes, stream, nullptr, nullptr, nullptr);
}

pqi_status pqi_tfim_sample_adj(const float* W, int n, const long long* adj_ptr, const int* adj_col,
                               const float* adj_val, const double* cum, double repulsion_base,
                               uint64_t seed, uint64_t round, int shots, uint32_t* theta_out,
                               void* workspace, size_t workspace_bytes, void* stream) {
  PQI_CHECK_ARG(adj_ptr && (adj_col || !adj_val) && (adj_val || !adj_col));
  return tfim_sample_impl(W, n, cum, repulsion_base, seed, round, shots, theta_out, workspace,
                          workspace_bytes, stream, adj_ptr, adj_col, adj_val);
}

pqi_status pqi_tfim_adj_count(const float* W, int n, long long* count, void* stream) {
  PQI_CHECK_ARG(W && count && n > 0);
  const int blocks = (int)std::min<long long>(((long long)n + 7) / 8, 148 * 16);
  tfim_adj_count_kernel<<<blocks, 256, 0, as_stream(stream)>>>(W, n, count);
  PQI_LAUNCHED("tfim_adj_count_kernel");
  return PQI_OK;
}

pqi_status pqi_tfim_adj_fill(const float* W, int n, const long long* adj_ptr, int* adj_col,
                             float* adj_val, void* stream) {
  PQI_CHECK_ARG(W && adj_ptr && n > 0);
  const int blocks = (int)std::min<long long>(((long long)n + 7) / 8, 148 * 16);
  tfim_adj_fill_kernel<<<blocks, 256, 0, as_stream(stream)>>>(W, n, adj_ptr, adj_col, adj_val);
  PQI_LAUNCHED("tfim_adj_fill_kernel");
  return PQI_OK;
}

}  // extern "C"
