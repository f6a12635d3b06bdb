/*
 * TEST INFRASTRUCTURE ONLY (oracle). Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load this; the product never does.
 *
 * Plain-C restatement of the dense OpenCL kernels of PyQrackIsing v9.16.6
 * (pyqrackising/kernels.cl) and of the host-side argmax that consumes them
 * (spin_glass_solver.py:156-307, maxcut_tfim.py:212-285). Floating-point sums
 * run in exactly the reference's order, one float32 rounding per add (build
 * with -ffp-contract=off), so float results are bit-identical to the
 * reference kernels when those are executed on the host (oracle/_ref).
 *
 * Parity-deciding behaviours restated here:
 *  - Selection (Q1): each work-item keeps the first strict maximum of its
 *    grid-stride sequence (kernels.cl:78-91); the work-group folds its items
 *    with the halving tree of reduce_energy_index (kernels.cl:1-29, strict
 *    '>' so ties keep the lower slot, and slots dropped by a non-power-of-two
 *    local size never reach slot 0); the host takes np.argmax over groups,
 *    i.e. the first group holding the maximum (spin_glass_solver.py:211).
 *  - Gray seeding (Q2): the seed mask uses a 32-bit int shift
 *    `1 << (offset & 63U)` (kernels.cl:925); OpenCL masks the count to 5 bits
 *    and a count of 31 yields INT_MIN, which sign-extends to
 *    0xFFFFFFFF80000000 when xor-ed into the 64-bit word.
 *  - Gray flips landing on k >= n (Q3) read outside W in the reference
 *    (kernels.cl:945-959). Here they are skipped (no flip, no energy) and
 *    counted in *oob so callers know when the reference is undefined.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline int bit32(const uint32_t* th, long u) { return (th[u >> 5] >> (u & 31)) & 1u; }
static inline int bit64(const uint64_t* th, long u) { return (int)((th[u >> 6] >> (u & 63)) & 1u); }

/* cut_worker, kernels.cl:44-62: upper-triangle sum, u-major then v. */
float orc_cut_one(const float* W, int n, const uint32_t* th, int is_spin_glass) {
  float e = 0.0f;
  for (int u = 0; u < n; ++u) {
    const float* row = W + (size_t)u * n;
    const int ub = bit32(th, u);
    for (int v = u + 1; v < n; ++v) {
      const float w = row[v];
      if (ub != bit32(th, v)) {
        e += w;
      } else if (is_spin_glass) {
        e -= w;
      }
    }
  }
  return e;
}

void orc_cut_values(const float* W, int n, const uint32_t* theta, int shots, int is_spin_glass,
                    float* out) {
  const int n32 = (n + 31) >> 5;
  /* candidates are independent: threads do not change any value */
#pragma omp parallel for schedule(dynamic, 1)
  for (int s = 0; s < shots; ++s) out[s] = orc_cut_one(W, n, theta + (size_t)s * n32, is_spin_glass);
}

/* single_bit_flip_worker, kernels.cl:100-116: the flipped bit against every
 * other bit, v ascending with v == k skipped. */
float orc_single_one(const float* W, int n, const uint32_t* th, int k) {
  const float* row = W + (size_t)k * n;
  const int kb = !bit32(th, k);
  float e = 0.0f;
  for (int v = 0; v < n; ++v) {
    if (v == k) continue;
    const float w = row[v];
    e += (kb == bit32(th, v)) ? -w : w;
  }
  return e;
}

/* Per-item values of single_bit_flips (kernels.cl:118-148), x2 for spin glass. */
void orc_single_values(const float* W, int n, const uint32_t* th, int is_spin_glass, float* out) {
  /* items are independent: threads do not change any value */
#pragma omp parallel for schedule(static)
  for (int k = 0; k < n; ++k) {
    float e = orc_single_one(W, n, th, k);
    if (is_spin_glass) e *= 2.0f;
    out[k] = e;
  }
}

/* double_bit_flip_worker, kernels.cl:150-184: both rows, interleaved per v,
 * v ascending with v in {k, l} skipped. */
float orc_double_one(const float* W, int n, const uint32_t* th, int k, int l) {
  if (l < k) {
    int t = k;
    k = l;
    l = t;
  }
  const float* rk = W + (size_t)k * n;
  const float* rl = W + (size_t)l * n;
  const int kb = !bit32(th, k), lb = !bit32(th, l);
  float e = 0.0f;
  for (int v = 0; v < n; ++v) {
    if (v == k || v == l) continue;
    const int vb = bit32(th, v);
    float w = rk[v];
    e += (kb == vb) ? -w : w;
    w = rl[v];
    e += (lb == vb) ? -w : w;
  }
  return e;
}

/* Linear pair index -> (k, l), kernels.cl:206-218 (k-major, l > k). */
void orc_pair_decode(int c, int n, int* k_out, int* l_out) {
  int k = 0, lcv = n - 1;
  while (c >= lcv) {
    c -= lcv;
    ++k;
    --lcv;
    if (!lcv) break;
  }
  *k_out = k;
  *l_out = c + k + 1;
}

/* reduce_energy_index tree (kernels.cl:1-29) over one group's L slots, in place.
 * Returns slot 0. */
static void group_tree(float* e, int* idx, int L) {
  for (int off = L >> 1; off > 0; off >>= 1) {
    for (int t = 0; t < off; ++t) {
      if (e[t + off] > e[t]) {
        e[t] = e[t + off];
        idx[t] = idx[t + off];
      }
    }
  }
}

/* Full selection over per-work-item maxima: group trees, then the host's
 * first-max over groups. thread_e/thread_i have G entries and are clobbered. */
static void fold_threads(float* thread_e, int* thread_i, int G, int L, float* best_e, int* best_i,
                         float* group_e, int* group_i) {
  const int groups = G / L;
  int bx = 0;
  for (int g = 0; g < groups; ++g) {
    group_tree(thread_e + (size_t)g * L, thread_i + (size_t)g * L, L);
    const float ge = thread_e[(size_t)g * L];
    const int gi = thread_i[(size_t)g * L];
    if (group_e) group_e[g] = ge;
    if (group_i) group_i[g] = gi;
    if (g == 0 || ge > thread_e[(size_t)bx * L]) bx = g;
  }
  *best_e = thread_e[(size_t)bx * L];
  *best_i = thread_i[(size_t)bx * L];
}

/* Generic selection over explicit values (count items) with ND-range (G, L).
 * group_e/group_i (G/L entries each) may be NULL. Returns 0, or -1 on a bad
 * geometry. */
int orc_select(const float* values, long count, int G, int L, float* best_e, int* best_i,
               float* group_e, int* group_i) {
  if (G <= 0 || L <= 0 || G % L) return -1;
  float* te = (float*)malloc(sizeof(float) * (size_t)G);
  int* ti = (int*)malloc(sizeof(int) * (size_t)G);
  for (int t = 0; t < G; ++t) {
    float be = -INFINITY;
    int bi = t;
    for (long i = t; i < count; i += G) {
      if (values[i] > be) {
        be = values[i];
        bi = (int)i;
      }
    }
    te[t] = be;
    ti[t] = bi;
  }
  fold_threads(te, ti, G, L, best_e, best_i, group_e, group_i);
  free(te);
  free(ti);
  return 0;
}

/* double_bit_flips (kernels.cl:186-231) end to end, values computed on the fly. */
int orc_double_select(const float* W, int n, const uint32_t* th, int is_spin_glass, int G, int L,
                      float* best_e, int* best_i) {
  if (G <= 0 || L <= 0 || G % L) return -1;
  const int combo = (int)(((long)n * (n - 1)) >> 1);
  float* te = (float*)malloc(sizeof(float) * (size_t)G);
  int* ti = (int*)malloc(sizeof(int) * (size_t)G);
  for (int t = 0; t < G; ++t) {
    float be = -INFINITY;
    int bi = t;
    for (int i = t; i < combo; i += G) {
      int k, l;
      orc_pair_decode(i, n, &k, &l);
      float e = orc_double_one(W, n, th, k, l);
      if (is_spin_glass) e *= 2.0f;
      if (e > be) {
        be = e;
        bi = i;
      }
    }
    te[t] = be;
    ti[t] = bi;
  }
  fold_threads(te, ti, G, L, best_e, best_i, NULL, NULL);
  free(te);
  free(ti);
  return 0;
}

/* Seed perturbation of the gray kernel for work-item gid (kernels.cl:915-926),
 * applied in place to a copy of theta (blocks 64-bit words). */
void orc_gray_seed(uint64_t* words, int n, long gid) {
  const uint64_t seed = (uint64_t)(gid ^ (gid >> 1));
  const int max_lcv = n < 64 ? n : 64;
  for (int b = 0; b < max_lcv; ++b) {
    if (!((seed >> (63 - b)) & 1u)) continue;
    const int offset = n - (b + 1);
    /* 32-bit int shift with the count masked to 5 bits, then sign-extended. */
    const int32_t m32 = (int32_t)(1u << ((unsigned)(offset & 63) & 31u));
    words[offset >> 6] ^= (uint64_t)(int64_t)m32;
  }
}

/* Gray-code walk of the gray kernel (kernels.cl:894-978) for all G work-items.
 * iters_bound is args[2] = ceil(gray_iterations / G). theta_out is G*blocks
 * words, energy_out is G floats. *oob counts flips skipped because k >= n.
 * margin_out (G floats, may be NULL) receives, per work-item, the smallest
 * |gain| over all of its keep-or-revert decisions (+inf if it made none): a
 * walk whose every decision clears a rounding bound is decided the same way
 * by any evaluation of the gains within that bound. Work-items are
 * independent, so they run on OpenMP threads without changing any value. */
void orc_gray_margin(const float* W, int n, const uint64_t* theta, int is_spin_glass,
                     int iters_bound, int G, uint64_t* theta_out, float* energy_out, long* oob,
                     float* margin_out) {
  const int blocks = (n + 63) >> 6;
  long skipped = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : skipped)
  for (int gid = 0; gid < G; ++gid) {
    uint64_t* loc = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)blocks);
    memcpy(loc, theta, sizeof(uint64_t) * (size_t)blocks);
    orc_gray_seed(loc, n, gid);
    float e = 0.0f;
    float margin = INFINITY;
    for (int u = 0; u < n; ++u) {
      const float* row = W + (size_t)u * n;
      const int ou = bit64(theta, u), nu = bit64(loc, u);
      for (int v = u + 1; v < n; ++v) {
        const int od = ou != bit64(theta, v);
        const int nd = nu != bit64(loc, v);
        if (od != nd) e += nd ? row[v] : -row[v];
      }
    }
    for (long i = gid; i < iters_bound; i += G) {
      const int c = __builtin_ctzl((unsigned long)(i + 1));
      for (int b = 0; b < blocks; ++b) {
        const long k = (long)c + ((long)b << 6);
        if (k >= n) {
          ++skipped;
          continue;
        }
        loc[k >> 6] ^= 1ull << (k & 63);
        const int kb = bit64(loc, k);
        const float* row = W + (size_t)k * n;
        float g = 0.0f;
        for (long v = 0; v < n; ++v) {
          if (v == k) continue;
          const float w = row[v];
          g += (kb == bit64(loc, v)) ? -w : w;
        }
        if (fabsf(g) < margin) margin = fabsf(g);
        if (g > 0.0f) {
          e += g;
        } else {
          loc[k >> 6] ^= 1ull << (k & 63);
        }
      }
    }
    memcpy(theta_out + (size_t)gid * blocks, loc, sizeof(uint64_t) * (size_t)blocks);
    if (!is_spin_glass) e /= 2;
    energy_out[gid] = e;
    if (margin_out) margin_out[gid] = margin;
    free(loc);
  }
  if (oob) *oob = skipped;
}

void orc_gray(const float* W, int n, const uint64_t* theta, int is_spin_glass, int iters_bound,
              int G, uint64_t* theta_out, float* energy_out, long* oob) {
  orc_gray_margin(W, n, theta, is_spin_glass, iters_bound, G, theta_out, energy_out, oob, NULL);
}

/* double_bit_flips selection (kernels.cl:186-231) with each pair value taken
 * from float64 single-flip gains: value(k, l) = g_k + g_l - 2 s_kl W_kl with
 * s_kl = +1 when bits k and l agree, else -1 (doubled for a spin glass),
 * rounded once to float32. For integer weights whose partial sums stay below
 * 2^24 this is exactly the reference's float32 sum over v, so the selected
 * (value, pair) is the reference's; it costs O(n^2) instead of O(n^3), which
 * makes full-size instances checkable. Pairs are visited in the reference's
 * k-major linear order and dealt to work-items by index modulo G. */
int orc_double_select_gains(const double* gains, const float* W, int n, const uint32_t* th,
                            int is_spin_glass, int G, int L, float* best_e, int* best_i) {
  if (G <= 0 || L <= 0 || G % L) return -1;
  float* te = (float*)malloc(sizeof(float) * (size_t)G);
  int* ti = (int*)malloc(sizeof(int) * (size_t)G);
  for (int t = 0; t < G; ++t) {
    te[t] = -INFINITY;
    ti[t] = t;
  }
  long c = 0;
  int t = 0;
  for (int k = 0; k < n; ++k) {
    const float* row = W + (size_t)k * n;
    const int kb = bit32(th, k);
    for (int l = k + 1; l < n; ++l, ++c) {
      const double sgn = (kb == bit32(th, l)) ? 1.0 : -1.0;
      double v = gains[k] + gains[l] - 2.0 * sgn * (double)row[l];
      if (is_spin_glass) v *= 2.0;
      const float e = (float)v;
      if (e > te[t]) {
        te[t] = e;
        ti[t] = (int)c;
      }
      if (++t == G) t = 0;
    }
  }
  fold_threads(te, ti, G, L, best_e, best_i, NULL, NULL);
  free(te);
  free(ti);
  return 0;
}
