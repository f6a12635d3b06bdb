/*
 * pqi.h - C ABI of libpqi, the B200 (sm_100a) implementation of PyQrackIsing's
 * dense cut-scoring and local-search path.
 *
 * Conventions
 *  - Every pointer argument is DEVICE memory owned by the caller unless the
 *    name ends in _host. The library never allocates or frees device memory;
 *    calls that need scratch take a caller-provided workspace whose size is
 *    given by pqi_workspace_bytes().
 *  - Every entry point returns a pqi_status. Launch errors are reported as
 *    PQI_ECUDA; a device-side iteration budget that runs out is PQI_ETIMEOUT.
 *  - `stream` is a cudaStream_t (NULL = legacy default stream). Calls are
 *    asynchronous on that stream unless documented otherwise.
 *  - Bit strings use the reference's layout: node j is bit (j & 31) of
 *    32-bit word (j >> 5) (pyqrackising/maxcut_tfim_util.py:304-316), or bit
 *    (j & 63) of 64-bit word (j >> 6) for the gray search (util:290-301).
 *  - Selection ("argmax") follows the reference's launch geometry
 *    (global_size G, local_size L as setup_opencl computes them,
 *    maxcut_tfim_util.py:169-221) so ties resolve to the same index as the
 *    reference: first maximum within each work-item's grid-stride sequence
 *    (kernels.cl:78-91), then the work-group halving tree of
 *    reduce_energy_index (kernels.cl:1-29), then the first group
 *    (np.argmax, spin_glass_solver.py:211). L must be <= 64 and divide G.
 */
#ifndef PQI_H
#define PQI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  PQI_OK = 0,
  PQI_EINVAL = 1,   /* bad argument: size, geometry, null pointer, unsupported weights */
  PQI_ECUDA = 2,    /* a CUDA launch or runtime call failed */
  PQI_ETIMEOUT = 3, /* a device-side iteration budget ran out; outputs are partial */
  PQI_ENOTSUP = 4   /* the device is not sm_100 or a feature is unavailable */
} pqi_status;

/* Storage chosen for the coupling matrix by pqi_prepare_weights. */
typedef enum {
  PQI_W_F32 = 0,  /* float32 only (non-integer weights) plus bf16 hi/lo split */
  PQI_W_I8 = 1    /* integer weights in [-127, 127]: exact int8 copy */
} pqi_wkind;

/*
 * Device-resident coupling matrix. W is n x n float32 row-major, symmetric,
 * as nx.to_numpy_array produces it (spin_glass_solver.py:458-461). The
 * prepared copies have a zero diagonal (the reference's kernels never read
 * the diagonal: kernels.cl:44-62, 100-116, 150-184). ld is the row pitch of
 * the prepared copies in elements (n rounded up to a multiple of 128), so
 * every prepared row starts on a 512-byte boundary.
 */
typedef struct {
  const float* W;        /* n*n float32, caller's matrix (diagonal as given) */
  const int8_t* W_i8;    /* n*ld int8 (PQI_W_I8), zero padded, else NULL */
  const uint16_t* W_hi;  /* n*ld bf16 bits (PQI_W_F32), zero padded, else NULL */
  const uint16_t* W_lo;  /* n*ld bf16 bits of W - hi (PQI_W_F32), else NULL */
  const float* W_f32z;   /* n*ld float32 with zero diagonal, zero padded */
  int n;
  int ld;
  int kind;              /* pqi_wkind */
  double upper_sum;      /* sum_{u<v} W_uv (host value, filled by pqi_prepare_weights) */
  const int8_t* W_d;     /* PQI_W_F32 (optional, pqi_prepare_digits): 4*n*ld int8, the
                            fixed-point digit planes of W_f32z, else NULL */
  double wscale;         /* W_f32z ~= wscale * (d0 2^24 + d1 2^16 + d2 2^8 + d3)
                            (pqi_prepare_digits) */
} pqi_weights;

/* ---------------------------------------------------------------------------
 * Set-up
 * -------------------------------------------------------------------------*/

/* Version string of the library build. */
const char* pqi_version(void);

/* Text of the last CUDA error the calling host thread saw inside the library. */
const char* pqi_last_error(void);

/* PQI_OK when device `device` is an sm_100 part the library was built for. */
pqi_status pqi_check_device(int device);

/* Bytes of workspace any entry point needs for a problem of n nodes and up
 * to `count` candidates / seeds. A workspace of this size serves every call. */
size_t pqi_workspace_bytes(int n, long count);

/* Row pitch (elements) of the prepared copies of an n-node matrix: W_f32z is
 * n*ld floats, W_i8 n*ld bytes, W_hi/W_lo n*ld bf16 each. */
int pqi_padded_ld(int n);

/* Result of pqi_scan_weights (host struct). */
typedef struct {
  unsigned long long nonfinite; /* NaN/Inf entries */
  unsigned long long nonint;    /* off-diagonal entries that are not integers */
  unsigned long long asym;      /* (i, j) with W_ij != W_ji, each pair counted twice */
  float maxabs;                 /* max |W_ij| off the diagonal */
  int kind;                     /* pqi_wkind the prepared copies will use */
  double upper_sum;             /* sum_{u<v} W_uv in float64 (fixed reduction order) */
} pqi_weight_stats;

/*
 * Scan W once on the device: finite, integer-valued, symmetric, max |W| and
 * the float64 sum of the upper triangle. Synchronises `stream` and fills
 * *stats_host. Returns PQI_EINVAL for non-finite or asymmetric W (the
 * reference's kernels read only the upper triangle for cuts but whole rows
 * for flips, so they agree only on symmetric matrices).
 */
pqi_status pqi_scan_weights(const float* W, int n, void* workspace, size_t workspace_bytes,
                            pqi_weight_stats* stats_host, void* stream);

/*
 * Build the prepared copies chosen by stats->kind: W_f32z always, W_i8 for
 * PQI_W_I8 (every off-diagonal weight an integer in [-127, 127]), W_hi/W_lo
 * for PQI_W_F32. Pointers of the copies not needed may be NULL. Fills
 * *out_host. Replaces make_G_m_buf (maxcut_tfim_util.py:224-238).
 */
pqi_status pqi_prepare_weights(const float* W, int n, const pqi_weight_stats* stats_host,
                               float* W_f32z, int8_t* W_i8, uint16_t* W_hi, uint16_t* W_lo,
                               pqi_weights* out_host, void* stream);

/*
 * Fixed-point digit planes of float weights, for exact tensor-core scoring:
 * W_f32z times 2^S (S the largest integer with maxabs * 2^S < 2^30 - 1) is
 * rounded to integers v, |v| < 2^30, and split into balanced int8 digits,
 * v = d0 2^24 + d1 2^16 + d2 2^8 + d3 (d in [-128, 127]); planes d0..d3 of
 * n*ld bytes each go to W_d (4*n*ld bytes). Fills w->W_d and w->wscale = 2^-S. The
 * scoring GEMM then accumulates each plane exactly in int32 and combines them
 * in 64-bit integers, so the only error of a score is the rounding of W to
 * multiples of 2^-S (at most 2^-S / 2 per weight). maxabs = max |W_ij| off the
 * diagonal (pqi_weight_stats.maxabs). No reference counterpart (the
 * reference sums float32 weights in float32).
 */
pqi_status pqi_prepare_digits(pqi_weights* w, float maxabs, int8_t* W_d, void* stream);

/* Select the batched-scoring implementation: 0 = tensor cores (tcgen05, the
 * default; CTA pairs with cta_group::2 MMAs for batches of more than 128
 * candidates, the +-1 operand expanded from the packed candidates by a
 * separate pass; float weights as their int8 digit planes when prepared, with
 * exact integer accumulation), 1 = CUDA cores, 2 = as 0 with single CTAs,
 * 3 = as 0, 4 = as 0 but float weights as split bf16 (hi + lo) with float32
 * accumulation, 5 = single CTAs that expand the packed candidates into their
 * operand tiles themselves (no expansion pass). Process-wide; used to
 * cross-check the implementations. */
pqi_status pqi_score_set_path(int path);

/* Record two caller-owned cudaEvent_t on the call's stream immediately before
 * and after the scoring GEMM launch inside each later pqi_calculate_cut (NULL,
 * NULL to stop). Process-wide; lets a caller time the GEMM kernel alone. */
pqi_status pqi_score_set_events(void* before, void* after);

/* Number of CTAs of the persistent tensor-core scoring kernel (0 = one per SM,
 * the default). Process-wide; a tuning knob for the scoring autotuner. */
pqi_status pqi_score_set_grid(int ctas);

/* ---------------------------------------------------------------------------
 * Kernel-level replacements of the reference's OpenCL kernels
 * -------------------------------------------------------------------------*/

/*
 * Batched cut scoring. theta: shots x ceil(n/32) words. Writes each
 * candidate's value, as cut_worker defines it (kernels.cl:44-62: sum over
 * u<v of W_uv if bits differ, else -W_uv when is_spin_glass, else 0), to
 * energies (float32, nullable), and the selected (value, index) under
 * geometry (G, L) to best_energy/best_index (device scalars). Integer
 * weights run on the int8 tensor-core path with int32 accumulation (exact);
 * float weights on the split-bf16 tensor-core path with fp32 accumulation.
 * If the tensor-core kernel gives up (a bounded wait expired), energies are
 * NaN and best_index is -1. Replaces calculate_cut (kernels.cl:64-94) plus the host argmax of
 * run_cut_opencl (maxcut_tfim.py:212-285).
 */
pqi_status pqi_calculate_cut(const pqi_weights* w, const uint32_t* theta, int shots,
                             int is_spin_glass, int global_size, int local_size,
                             float* energies, float* best_energy, int* best_index,
                             void* workspace, size_t workspace_bytes, void* stream);

/*
 * Single-flip gain vectors for `count` states: gains[b*n + k] = the cut change
 * of flipping node k of state b, i.e. sum_{v != k} W_kv * (s_k == s_v ? 1 : -1)
 * (single_bit_flip_worker, kernels.cl:100-116). float32 output; gains64
 * (nullable) receives the same values accumulated in float64.
 */
pqi_status pqi_gains(const pqi_weights* w, const uint32_t* theta, int count, float* gains,
                     double* gains64, void* workspace, size_t workspace_bytes, void* stream);

/*
 * Selection over `count` float32 values under geometry (G, L); NaN never
 * selected. Writes device scalars best_value/best_index.
 * Replaces reduce_energy_index (kernels.cl:1-29) plus np.argmax over groups.
 */
pqi_status pqi_select(const float* values, long count, int global_size, int local_size,
                      float* best_value, int* best_index, void* workspace,
                      size_t workspace_bytes, void* stream);

/*
 * Host twin of pqi_select over host memory (no GPU needed): the same 64-bit
 * key order, evaluated on the CPU. For callers that select on the host and
 * for checking the key order against the reference's reduction.
 */
pqi_status pqi_select_host(const float* values_host, long count, int global_size, int local_size,
                           float* best_value_host, int* best_index_host);

/*
 * One single-bit-flip pass: value_k = gain_k (x2 when is_spin_glass), selected
 * under (G, L). Replaces single_bit_flips (kernels.cl:118-148).
 */
pqi_status pqi_single_bit_flips(const pqi_weights* w, const uint32_t* theta, int is_spin_glass,
                                int global_size, int local_size, float* best_energy,
                                int* best_index, void* workspace, size_t workspace_bytes,
                                void* stream);

/* Largest n pqi_single_bit_flips_noalloc accepts, and the bytes of the device
 * array it uses in place of a workspace (a selection key, then n floats). */
#define PQI_NOALLOC_MAX_N 65536
#define PQI_NOALLOC_BYTES (256 + 4 * PQI_NOALLOC_MAX_N)

/*
 * pqi_single_bit_flips without a workspace, for callers that cannot allocate
 * device memory: a process whose device memory belongs to another framework's
 * allocator, or a loop that must not call cudaMalloc because it can synchronise
 * the device. No counterpart in the reference (its OpenCL host glue allocates
 * buffers on every call, maxcut_tfim_util.py:169-221).
 * Scratch is one array of PQI_NOALLOC_BYTES compiled into the library, held by
 * every GPU that loads it until exit. The first call on a device looks up that
 * array's device address (cudaGetSymbolAddress, with the device current); make
 * it before any stream capture. All calls share the array, which keeps the last
 * call's contents: calls that overlap on the GPU race. Allocates nothing.
 * The looked-up address is kept per device ordinal for the life of the
 * process, so this call serves the device's primary context (the runtime
 * API's) and must not be used after cudaDeviceReset on that device.
 * Returns PQI_EINVAL when n > PQI_NOALLOC_MAX_N (pqi_last_error() says so).
 * Same outputs as pqi_single_bit_flips.
 */
pqi_status pqi_single_bit_flips_noalloc(const pqi_weights* w, const uint32_t* theta,
                                        int is_spin_glass, int global_size, int local_size,
                                        float* best_energy, int* best_index, void* stream);

/*
 * One double-bit-flip pass over all pairs k < l in the reference's linear
 * order c = k(n-1) - k(k-1)/2 + (l-k-1) (kernels.cl:206-218): value_c =
 * g_k + g_l - 2 W_kl (s_k == s_l ? 1 : -1), x2 when is_spin_glass, which equals
 * double_bit_flip_worker (kernels.cl:150-184). gains64 (nullable) are the
 * float64 gains of theta from pqi_gains; when NULL they are computed here.
 * best_index receives c. Replaces double_bit_flips (kernels.cl:186-231).
 * n(n-1)/2 must fit in int32, as in the reference (n <= 46341).
 */
pqi_status pqi_double_bit_flips(const pqi_weights* w, const uint32_t* theta,
                                const double* gains64, int is_spin_glass, int global_size,
                                int local_size, float* best_energy, int* best_index,
                                void* workspace, size_t workspace_bytes, void* stream);

/*
 * Parallel Gray-code search of `seeds` perturbed copies of theta64
 * (ceil(n/64) words), with the reference's schedule (gray kernel,
 * kernels.cl:894-978): seed s starts from theta xor the seed mask of work-item
 * s (kernels.cl:915-926, including its 32-bit shift), then for i = s, s+seeds,
 * ... < iters_bound and every 64-node block b flips node ctz(i+1) + 64b and
 * keeps the flip when it raises the cut. Flips landing on a node >= n are
 * skipped (the reference reads outside W there). Writes theta_out
 * (seeds x ceil(n/64) words) and energy_out (seeds floats: cut change of the
 * seed's final state, halved when !is_spin_glass, as kernels.cl:974-976).
 * gains64 (nullable): float64 gains of theta. Gains are kept per seed in
 * shared memory and updated in O(n) per accepted flip instead of recomputed.
 * Replaces gray (kernels.cl:894-978).
 */
pqi_status pqi_gray(const pqi_weights* w, const uint64_t* theta64, const double* gains64,
                    int is_spin_glass, int iters_bound, int seeds, uint64_t* theta_out,
                    float* energy_out, void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------------
 * Device-resident search (no host round trip per accepted move)
 * -------------------------------------------------------------------------*/

/*
 * Repeats single-bit-flip passes on the device until no flip has positive
 * value or max_flips flips were made: each step selects under (G, L) exactly
 * as pqi_single_bit_flips and, if the value is > 0, flips that node and
 * updates the gains in O(n). theta (in/out, ceil(n/32) words) and gains64
 * (in/out, float64, from pqi_gains) stay on the device. Outputs (device):
 * energy_sum (float64 sum of the accepted float32 values, what the
 * reference adds to max_energy at spin_glass_solver.py:623-626), flips
 * (int), and trace (nullable, max_flips ints: the flipped nodes in order).
 * Returns PQI_ETIMEOUT when max_flips is reached with an improving flip left.
 * Replaces the repeated single-flip iterations of the driver loop
 * (spin_glass_solver.py:605-627).
 */
pqi_status pqi_single_descent(const pqi_weights* w, uint32_t* theta, double* gains64,
                              int is_spin_glass, int global_size, int local_size, int max_flips,
                              double* energy_sum, int* flips, int* trace, void* workspace,
                              size_t workspace_bytes, void* stream);

/* Flip nodes k (and l when l >= 0) of theta and update gains64 in O(n).
 * Used after an accepted double flip or to apply a move chosen on the host. */
pqi_status pqi_apply_flip(const pqi_weights* w, uint32_t* theta, double* gains64, int k, int l,
                          void* stream);

/*
 * Exhaustive search over all 2^n states (1 <= n <= 30; the reference uses it
 * for n < 24). W is the caller's n*n float32 matrix. Values are float64 sums in
 * the reference's order: exact_maxcut sums W_ij over i<j with differing bits,
 * exact_spin_glass sums +W_ij for equal bits and -W_ij otherwise
 * (maxcut_tfim.py:288-339). Writes the reference's selection: the smallest
 * mask attaining the maximum when that exceeds -1.0, else (mask 0, -1.0).
 * best_value (double) and best_mask (int, bit i = node i) are device scalars.
 */
pqi_status pqi_exact_search(const float* W, int n, int is_spin_glass, double* best_value,
                            int* best_mask, void* workspace, size_t workspace_bytes,
                            void* stream);

/* ---------------------------------------------------------------------------
 * Batched local search (many graphs x many starting states, one launch)
 * -------------------------------------------------------------------------*/

/* Size of one graph descriptor in the device array pqi_batch_search reads:
 * {const void* W (prepared W_i8 or W_f32z); int n; int ld; int kind; int pad;
 *  double upper_sum; const long long* adj_ptr; const int* adj_col;
 *  const float* adj_val} -- the last three the row lists of a sparse graph's
 * nonzero weights (pqi_tfim_adj_count / pqi_tfim_adj_fill; the diagonal may be
 * listed and is skipped), used for the starting fields, or null. */
size_t pqi_batch_graph_desc_bytes(void);

/*
 * Iterated local search for `tasks` (graph, starting state) pairs in one
 * persistent launch. Task t uses graph task_graph[t] and starts from
 * init_states + t*words_pitch (ceil(n/32) words). Per task: rounds+1 steepest
 * single-flip ascents (largest gain, lowest node on ties, while > 0, at most
 * flip_budget flips each) separated by `kick` forced flips per round, drawn
 * uniformly or, when kick_cdf is given, from the graph's proposal distribution
 * (normalised cumulative array at kick_cdf + cdf_offset[graph]). Writes the
 * best state (best_states + t*words_pitch) and value (cut, or the spin energy
 * sum_{u<v} W_uv (s_u != s_v ? 1 : -1) when is_spin_glass) of each task, adds
 * the flips made to *flips_total and sets *status to PQI_ETIMEOUT if a flip
 * budget ran out. All graphs of a launch share `kind`; max_n bounds their n.
 * No reference counterpart: it batches the single-graph loop of
 * spin_glass_solver.py:603-717.
 */
pqi_status pqi_batch_search(const void* graphs, int num_graphs, const int* task_graph,
                            const uint32_t* init_states, int words_pitch, int tasks, int max_n,
                            int kind, int is_spin_glass, int rounds, int kick, int flip_budget,
                            uint64_t seed, const double* kick_cdf, const long long* cdf_offset,
                            uint32_t* best_states, double* best_values,
                            unsigned long long* flips_total, int* status, void* stream);

/*
 * pqi_batch_search with float32 local fields for float-weight graphs (int8
 * graphs are unchanged: their fields are exact int32). Half the shared memory
 * and fewer registers per task, so four tasks are resident per SM instead of
 * three; the gains are float32 (as the reference's), the running value and the
 * returned values stay float64 sums of exact-to-float32 gains. Field rounding
 * can change the trajectory against the float64-field form. No reference
 * counterpart.
 */
pqi_status pqi_batch_search_f32(const void* graphs, int num_graphs, const int* task_graph,
                                const uint32_t* init_states, int words_pitch, int tasks,
                                int max_n, int kind, int is_spin_glass, int rounds, int kick,
                                int flip_budget, uint64_t seed, const double* kick_cdf,
                                const long long* cdf_offset, uint32_t* best_states,
                                double* best_values, unsigned long long* flips_total,
                                int* status, void* stream);

/* pqi_batch_search (float32_fields 0) or pqi_batch_search_f32 (1) with the
 * CTA size given: threads_per_task 256 (those entry points' size), 128 or 64
 * (two or four times the resident tasks per SM at the same registers per
 * thread; for graphs of up to a few thousand nodes). Same results for every
 * size. No reference counterpart (batched form of spin_glass_solver.py:603-717). */
pqi_status pqi_batch_search_cta(const void* graphs, int num_graphs, const int* task_graph,
                                const uint32_t* init_states, int words_pitch, int tasks,
                                int max_n, int kind, int is_spin_glass, int rounds, int kick,
                                int flip_budget, uint64_t seed, const double* kick_cdf,
                                const long long* cdf_offset, uint32_t* best_states,
                                double* best_values, unsigned long long* flips_total,
                                int* status, int threads_per_task, int float32_fields,
                                void* stream);

/* Tuning / cross-check knob (no reference counterpart): on (default) lets
 * pqi_batch_search_f32 (float32 local fields) stage four row groups per thread
 * in shared memory with cp.async for graphs of more than 4096 nodes; off keeps
 * every row group in registers. Results are identical. */
pqi_status pqi_batch_set_staging(int on);

/* Tuning / cross-check knob (no reference counterpart): on (default) lets
 * pqi_batch_search (float64 local fields, CTA form) keep the fields of float
 * graphs of 4097 to 16384 nodes in tensor memory (four tasks per SM up to 8192
 * nodes, two up to 16384), each flip's row fetched whole by one bulk copy; off
 * keeps them in shared memory (three tasks per SM up to 8192 nodes, one up to
 * 16384). Results are identical. */
pqi_status pqi_batch_set_tmem_fields(int on);

/* Cross-check knob (no reference counterpart): on (default) the batched
 * searches and the cluster ascent of graphs of 64 nodes or more compute the
 * starting local fields of all dense-graph tasks first, one pass over W per
 * tile of 64 tasks x 64 nodes (float64 sums, u ascending: the search
 * kernels' own order), into a buffer from the device's stream-ordered memory
 * pool; off, every task sums its own fields from W. */
pqi_status pqi_batch_set_start_pass(int on);

/*
 * pqi_batch_search with one warp per task instead of one CTA: the same search,
 * selection rule, kick stream, outputs and status, for graphs with
 * max_n <= 1024. Fields and bits live in registers (no shared memory, no
 * block barrier), so many more tasks are in flight per SM. warps_per_sm caps
 * the resident warps per SM (0 = as many as fit). No reference counterpart
 * (batched form of spin_glass_solver.py:603-717).
 */
pqi_status pqi_batch_search_warp(const void* graphs, int num_graphs, const int* task_graph,
                                 const uint32_t* init_states, int words_pitch, int tasks,
                                 int max_n, int kind, int is_spin_glass, int rounds, int kick,
                                 int flip_budget, uint64_t seed, const double* kick_cdf,
                                 const long long* cdf_offset, uint32_t* best_states,
                                 double* best_values, unsigned long long* flips_total,
                                 int* status, int warps_per_sm, void* stream);

/*
 * Steepest single-flip ascent (rounds = 0 of pqi_batch_search: same selection
 * rule, same trajectory, same outputs and status) with one thread-block
 * cluster of cluster_size CTAs (2, 4, 8 or 16) per task: the task's nodes are
 * split over the cluster's CTAs, whose local fields stay on chip, and the
 * per-flip argmax is exchanged through distributed shared memory. Lower
 * latency per flip than one CTA per task for large n; max_n must satisfy
 * ceil(max_n / cluster_size) <= 8192 nodes per CTA. No reference counterpart:
 * it is the single-flip descent of spin_glass_solver.py:603-717 on a cluster.
 * reached (device int, zeroed by the caller; NULL for none): target mode.
 * A task whose running value is >= target sets *reached = 1 (checked every
 * 16 flips and at the task's end), and every task stops at its next 16-flip
 * check once the flag is set, so the launch ends soon after the first task
 * reaches the target. best_states / best_values hold each task's state and
 * value where it stopped (status stays 0 for such a stop).
 */
pqi_status pqi_cluster_ascent(const void* graphs, int num_graphs, const int* task_graph,
                              const uint32_t* init_states, int words_pitch, int tasks, int max_n,
                              int kind, int is_spin_glass, int cluster_size, int flip_budget,
                              uint32_t* best_states, double* best_values,
                              unsigned long long* flips_total, int* status, double target,
                              int* reached, void* stream);

/* ---------------------------------------------------------------------------
 * Learned flip-proposal network (no reference counterpart). bf16 storage,
 * float32 accumulation. Pointers typed void* hold bf16 (__nv_bfloat16) data.
 * -------------------------------------------------------------------------*/

/* C[M x N] = alpha op(A) op(B) + beta C32 + bias, optional ReLU; op(X) = X^T when
 * the trans flag is set (A is then K x M with pitch lda, B is N x K with pitch
 * ldb). Writes C32 (float32) and/or C16 (bf16) with pitch ldc. */
pqi_status pqi_mpnn_gemm(int transA, int transB, int M, int N, int K, float alpha, const void* A,
                         int lda, const void* B, int ldb, float beta, float* C32, void* C16,
                         int ldc, const float* bias, int relu, void* stream);

/* OUT[:, 0:64] = A_hat X (+ beta * OUT32) on the tensor cores (tcgen05,
 * bf16 operands, float32 accumulation): A_hat is n x n bf16 with pitch ld, X
 * is given transposed (Xt: 64 x n bf16, pitch ldt); writes OUT32 (float32)
 * and / or OUT16 (bf16), row pitch ldo. ld and ldt multiples of 8, 16-byte
 * aligned bases. PQI_ENOTSUP off sm_100. */
pqi_status pqi_mpnn_adj_gemm(const void* Ahat, int ld, int n, const void* Xt, int ldt, float beta,
                             float* out32, void* out16, int ldo, void* stream);

/* Xt[c][r] = X[r][c] for r < n, c < 64 (bf16; X pitch ldx >= 64, Xt pitch
 * ldt >= n, rows n..ldt-1 of Xt zeroed). */
pqi_status pqi_mpnn_transpose64(const void* X, int n, int ldx, void* Xt, int ldt, void* stream);

/* A_hat = D^-1/2 W D^-1/2 in bf16 (n x ld, zero diagonal and padding) and
 * s_v = sum_{u != v} |W_vu| (float32) from the caller's n x n W. */
pqi_status pqi_mpnn_norm_adj(const float* W, int n, void* Ahat, int ld, float* s, void* stream);

/* Node features of a state, bf16 n x 4: [x_v, g_v / s_v, s_v / mean_s, 1]. */
pqi_status pqi_mpnn_features(const uint32_t* theta, const double* gains64, const float* s,
                             float mean_s, int n, void* F, void* stream);

/* Gradient clipping: *norm_out (nullable) = the L2 norm of g (float64
 * accumulation); when it exceeds max_norm > 0, g is scaled to max_norm. */
pqi_status pqi_mpnn_grad_clip(float* g, size_t count, float max_norm, float* norm_out, void* stream);

/* *out = sum of count floats, float64, fixed order (one block). */
pqi_status pqi_mpnn_sum(const float* x, size_t count, double* out, void* stream);

/* Kick distributions of `tasks` states from their logits (tasks x n,
 * contiguous): softmax(logit / temperature) in float64, mixed with the
 * uniform distribution ((1 - mix) p + mix / n), as normalised cumulative
 * arrays (tasks x n float64, the batched search's kick_cdf). A task with a
 * non-finite logit gets the uniform distribution. */
pqi_status pqi_mpnn_kick_cdf(const float* logits, int n, int tasks, float temperature, float mix,
                             double* cdf, void* stream);

/* Softmax of n logits: *loss = -sum_v t_v log p_v, dlogits = p - t, prob = p
 * (each output and target nullable). One block. */
pqi_status pqi_mpnn_softmax_xent(const float* logits, const float* target, int n, float* loss,
                                 float* dlogits, float* prob, void* stream);

/* dZ = dY * (Y > 0) (Y the ReLU output), float32 and optional bf16 copy. */
pqi_status pqi_mpnn_relu_bwd(const float* dY, const float* Y, size_t count, float* dZ, void* dZ16,
                             void* stream);

/* out[c] (+)= sum over rows of X[r*ld + c] (bias gradients). */
pqi_status pqi_mpnn_colsum(const float* X, int rows, int cols, int ld, float* out,
                           int accumulate, void* stream);

/* float32 -> bf16. */
pqi_status pqi_mpnn_to_bf16(const float* x, size_t count, void* y, void* stream);

/* One Adam step on float32 master weights w (bias-corrected, step >= 1), with
 * a bf16 copy written to w16 (nullable). */
pqi_status pqi_mpnn_adam(float* w, const float* g, float* m, float* v, void* w16, size_t count,
                         float lr, float b1, float b2, float eps, int step, void* stream);

/* ---------------------------------------------------------------------------
 * TFIM-inspired candidate sampler of maxcut_tfim
 * -------------------------------------------------------------------------*/

/* Per-node J_eff (float64) and degree (uint32) of the caller's n*n W, as
 * init_J_and_z (maxcut_tfim.py:189-209): an entry counts when W_ij - min(W) >
 * FLT_EPSILON (float32 difference), J_eff = -(sum of those differences)/degree. */
pqi_status pqi_tfim_jz(const float* W, int n, double* J_eff, unsigned int* degrees,
                       void* workspace, size_t workspace_bytes, void* stream);

/* pqi_tfim_jz with the reference's sparse-path arithmetic
 * (maxcut_tfim_sparse.py:204-224, plain numpy scalars): float32 row sums in
 * node order and a float32 division. W is the dense matrix of the stored
 * (upper-triangular) entries. */
pqi_status pqi_tfim_jz_f32(const float* W, int n, double* J_eff, unsigned int* degrees,
                           void* workspace, size_t workspace_bytes, void* stream);

/* Dense matrices of a sparse graph's stored entries (rows[e], cols[e], vals[e]),
 * e < nnz, coordinates unique: S = the stored off-diagonal entries, W = S + S^T
 * (both n*n float32 row-major, zeroed by the call; S nullable). Replaces the
 * reference's CSR handling of the sparse entry points
 * (maxcut_tfim_util.py:533-542 builds the CSR; kernels.cl:233-251 sums over it
 * as W): the dense path then runs on W, the sampler's J / degrees on S. An
 * out-of-range coordinate is skipped and sets *bad (device int) to 1. */
pqi_status pqi_coo_to_dense(const int* rows, const int* cols, const float* vals, long long nnz,
                            int n, float* S, float* W, int* bad, void* stream);

/* One batch of branch-and-bound frontier nodes of the exact solver
 * (solve_maxcut_bnb.py:47-121, called from the loop of :128-199). fixed_t holds
 * the nodes' assignments node-minor: entry i of node b at fixed_t[i * count + b]
 * (-1 free, 0 / 1 fixed). W is the caller's n*n float32 matrix (upper triangle
 * read). Per node, in the reference's summation order: ub[b] = the decoupled
 * upper bound; state[b] = 0 when ub[b] <= best_value + 1e-9 (pruned), else 1 for a
 * leaf with leaf_value[b] = its cut (is_spin_glass 0) or energy (1), else 2 with
 * branch_var[b] = the first free variable of largest free-to-free |W| sum. */
pqi_status pqi_bnb_eval(const float* W, int n, const int8_t* fixed_t, int count, double best_value,
                        int is_spin_glass, double* ub, double* leaf_value, int* branch_var,
                        int8_t* state, void* stream);

/* Workspace bytes pqi_tfim_cdf needs. */
size_t pqi_tfim_cdf_workspace_bytes(int n, int quality);

/* Cumulative Hamming-weight distribution, n-1 float64 entries, as
 * maxcut_hamming_cdf (maxcut_tfim_util.py:654-687) with
 * probability_by_hamming_weight and _apply_time_envelope (util:578-651);
 * thresholds (n+1 float64, init_thresholds of util:558-575) seed the sum. */
pqi_status pqi_tfim_cdf(const double* J_eff, const unsigned int* degrees, int n, int quality,
                        double anneal_t, double anneal_h, const double* thresholds, double* cum,
                        void* workspace, size_t workspace_bytes, void* stream);

/* Workspace bytes pqi_tfim_sample needs for n nodes (large n only). */
size_t pqi_tfim_sample_workspace_bytes(int n);

/* Draw `shots` candidates as packed bits (shots x ceil(n/32) words): shot s
 * draws a Hamming-weight index from `cum` (sample_mag, util:691-707) and picks
 * nodes starting at s % n with weights multiplied by repulsion_base^(-W_kv)
 * after each pick (local_repulsion_choice, maxcut_tfim.py:36-74; bit_pick,
 * util:711-724); selected = weight exactly zero. Random draws are a
 * counter-based function of (seed, round, s, draw). */
pqi_status pqi_tfim_sample(const float* W, int n, const double* cum, double repulsion_base,
                           uint64_t seed, uint64_t round, int shots, uint32_t* theta_out,
                           void* workspace, size_t workspace_bytes, void* stream);

/* pqi_tfim_sample with the nonzero entries of W's rows as lists (row r's
 * columns adj_col[adj_ptr[r] .. adj_ptr[r+1]) ascending, values adj_val, from
 * pqi_tfim_adj_count / pqi_tfim_adj_fill): a repulsion update
 * (maxcut_tfim.py:37-45) walks the picked node's list instead of scanning its
 * row. The same multiplications in the same order: the same draws, bit for bit. */
pqi_status pqi_tfim_sample_adj(const float* W, int n, const long long* adj_ptr, const int* adj_col,
                               const float* adj_val, const double* cum, double repulsion_base,
                               uint64_t seed, uint64_t round, int shots, uint32_t* theta_out,
                               void* workspace, size_t workspace_bytes, void* stream);

/* Nonzero count of each row of the n*n float32 W (count: n int64, device). */
pqi_status pqi_tfim_adj_count(const float* W, int n, long long* count, void* stream);

/* Row lists of W's nonzero entries in column order: row r at adj_ptr[r] (n + 1
 * int64, the exclusive prefix sum of the counts), columns into adj_col, values
 * into adj_val. */
pqi_status pqi_tfim_adj_fill(const float* W, int n, const long long* adj_ptr, int* adj_col,
                             float* adj_val, void* stream);

/* ---------------------------------------------------------------------------
 * Objectives, packing
 * -------------------------------------------------------------------------*/

/*
 * float64 re-scoring of `count` states (ceil(n/32) words each) against the
 * caller's W (diagonal included, as compute_cut / compute_energy,
 * maxcut_tfim_util.py:319-331): cut[b] = 1/2 sum_{u,v} W_uv [s_u != s_v],
 * energy[b] = 1/2 sum_{u,v} W_uv (2[s_u != s_v] - 1). Either output nullable.
 * Deterministic (fixed reduction order).
 */
pqi_status pqi_rescore_fp64(const pqi_weights* w, const uint32_t* theta, int count, double* cut,
                            double* energy, void* workspace, size_t workspace_bytes,
                            void* stream);

/* bools (rows x n bytes, nonzero = 1) -> words (rows x ceil(n/32) uint32).
 * Replaces convert_bool_to_uint (maxcut_tfim_util.py:304-316). */
pqi_status pqi_pack_bits(const uint8_t* bools, int rows, int n, uint32_t* words, void* stream);

/* words (rows x ceil(n/32)) -> bytes 0/1 (rows x n). */
pqi_status pqi_unpack_bits(const uint32_t* words, int rows, int n, uint8_t* bools, void* stream);

/* ---------------------------------------------------------------------------
 * Sparse graphs: the coupling matrix in compressed rows (CSR), O(n + nnz)
 * device memory, for graphs too large to hold as an n x n matrix. Replaces
 * the reference's CSR kernels (kernels.cl:233-414, 1072-1150) and buffers
 * (make_G_m_csr_buf, spin_glass_solver_sparse.py:659-661). Every entry point
 * has the semantics of its dense counterpart above (same values, same
 * reference-order selection); a flip costs O(degree).
 * -------------------------------------------------------------------------*/

/* Both triangles stored: row r lists every neighbour c != r once, columns
 * ascending, with val = W_rc = W_cr. ptr has n + 1 entries (ptr[0] = 0,
 * ptr[n] = nnz). */
typedef struct {
  const long long* ptr;
  const int* col;
  const float* val;
  int n;
  int pad;
  long long nnz;
  double upper_sum; /* sum over edges u < v of W_uv (float64, host value) */
} pqi_csr;

/* Gains of `count` states (rows of ceil(n/32) words): g_k = sum over
 * neighbours v of W_kv (s_k == s_v ? +1 : -1), float64 (and/or float32).
 * Replaces the sums of single_bit_flips_sparse (kernels.cl:253-283). */
pqi_status pqi_csr_gains(const pqi_csr* g, const uint32_t* theta, int count, float* g32,
                         double* g64, void* stream);

/* pqi_single_bit_flips on CSR (kernels.cl:233-283 with the host argmax). */
pqi_status pqi_csr_single_bit_flips(const pqi_csr* g, const uint32_t* theta, int is_spin_glass,
                                    int global_size, int local_size, float* best_energy,
                                    int* best_index, void* workspace, size_t workspace_bytes,
                                    void* stream);

/* pqi_apply_flip on CSR: O(degree) per flipped node. */
pqi_status pqi_csr_apply_flip(const pqi_csr* g, uint32_t* theta, double* gains64, int k, int l,
                              void* stream);

/* pqi_single_descent on CSR (one CTA; gains updated in place in gains64).
 * Synchronises `stream`; returns PQI_ETIMEOUT when max_flips runs out. */
pqi_status pqi_csr_single_descent(const pqi_csr* g, uint32_t* theta, double* gains64,
                                  int is_spin_glass, int global_size, int local_size,
                                  int max_flips, double* energy_sum, int* flips, int* trace,
                                  void* workspace, size_t workspace_bytes, void* stream);

/* pqi_double_bit_flips on CSR over all n(n-1)/2 pairs (kernels.cl:285-414
 * semantics): the pair index c = k(n-1) - k(k-1)/2 + (l-k-1) is 64-bit
 * (best_index), so n above 46341, where the reference's int32 pair count
 * overflows, has a defined result (the same rule with 64-bit indices).
 * gains64 nullable (computed here when NULL). */
pqi_status pqi_csr_double_bit_flips(const pqi_csr* g, const uint32_t* theta, const double* gains64,
                                    int is_spin_glass, int global_size, int local_size,
                                    float* best_energy, long long* best_index, void* workspace,
                                    size_t workspace_bytes, void* stream);

/* pqi_csr_double_bit_flips for a caller that applies the selected pair only
 * when its value is > 0 (the solver loop, spin_glass_solver_sparse.py:727-751):
 * whenever the best pair value is > 0, the same best_energy and best_index;
 * otherwise best_energy <= 0 (-inf allowed) and best_index is -1 or a pair of
 * that value. Pairs whose fp32 estimate is not > 0 are never scored, so at a
 * single-flip local optimum (every gain <= 0) only the adjacent pairs are.
 * Same arguments and workspace. No reference counterpart (an early-out of the
 * reference's own loop). */
pqi_status pqi_csr_improving_double_flip(const pqi_csr* g, const uint32_t* theta,
                                         const double* gains64, int is_spin_glass,
                                         int global_size, int local_size, float* best_energy,
                                         long long* best_index, void* workspace,
                                         size_t workspace_bytes, void* stream);

/* pqi_gray on CSR (the gray_sparse kernel's schedule, kernels.cl:1072-1150);
 * gains64 required. Workspace: n float64 per resident seed. */
pqi_status pqi_csr_gray(const pqi_csr* g, const uint64_t* theta64, const double* gains64,
                        int is_spin_glass, long long iters_bound, int seeds, uint64_t* theta_out,
                        float* energy_out, void* workspace, size_t workspace_bytes, void* stream);

/* float64 cut and energy of `rows` states (compute_cut_sparse /
 * compute_energy_sparse, maxcut_tfim_util.py:349-372, on the symmetric rows). */
pqi_status pqi_csr_rescore_fp64(const pqi_csr* g, const uint32_t* words, int rows, double* cut,
                                double* energy, void* stream);

/* The TFIM sampler's J_eff and degrees from the stored rows S (CSR as the
 * caller stores them, columns ascending; the entries absent from a row are
 * zeros) with the reference's sparse-path arithmetic (maxcut_tfim_sparse.py:
 * 204-224; pqi_tfim_jz_f32 on the dense S gives the same values). gmin =
 * min over all of S, zeros included. */
pqi_status pqi_csr_tfim_jz(const long long* ptr, const int* col, const float* val, int n, float gmin,
                           double* J_eff, unsigned int* degrees, void* stream);

/* pqi_calculate_cut on CSR (calculate_cut_sparse semantics): values of `shots`
 * candidates, O(nnz) each, then the reference-order selection. */
pqi_status pqi_csr_calculate_cut(const pqi_csr* g, const uint32_t* theta, int shots,
                                 int is_spin_glass, int global_size, int local_size,
                                 float* energies, float* best_energy, int* best_index,
                                 void* workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PQI_H */
