/*
 * TEST INFRASTRUCTURE ONLY (oracle). Never linked into the product library.
 *
 * A host-side ND-range emulator for the reference's dense OpenCL kernels
 * (pyqrackising/kernels.cl), compiled from the reference source where it lies
 * by oracle/build_ref.sh into oracle/_ref/libpqi_ref.so.
 *
 * Each work-group runs as L POSIX threads (L = local size, <= 32 on the
 * reference's launch shapes, maxcut_tfim_util.py:169-221) that share one
 * pthread barrier, so reduce_energy_index (kernels.cl:1-29) executes with its
 * real barrier semantics. Work-groups run concurrently, in waves of up to 256
 * work-items (every group with its own barrier and local arrays), which is a
 * legal OpenCL schedule because the kernels do not communicate across groups.
 *
 * The launch arguments mirror the host glue of the reference:
 *   calculate_cut     args = [n, shots, is_spin_glass, seg, theta_seg]  (maxcut_tfim.py:167-171)
 *   single/double     args = [n, is_spin_glass, seg]                     (spin_glass_solver.py:571-575)
 *   gray              args = [n, is_spin_glass, ceil(iters/G), seg]      (spin_glass_solver.py:586-600)
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "ref_shim.h"

/* Kernels defined in kernels.cl. */
void calculate_cut(const float* G_m, uint* theta, const int* args, float* max_energy_ptr,
                   int* max_index_ptr, float* loc_energy, int* loc_index);
void single_bit_flips(const float* G_m, const uint* best_theta, const int* args,
                      float* max_energy_ptr, int* max_index_ptr, float* loc_energy,
                      int* loc_index);
void double_bit_flips(const float* G_m, const uint* best_theta, const int* args,
                      float* max_energy_ptr, int* max_index_ptr, float* loc_energy,
                      int* loc_index);
void gray(const float* G_m, const ulong* theta, const int* args, ulong* theta_out,
          float* energy_out);

static __thread size_t tl_gid, tl_lid, tl_grp, tl_gsize, tl_lsize;
static __thread pthread_barrier_t* tl_bar;

size_t pqi_ref_get_global_id(uint d) { return d == 0 ? tl_gid : 0; }
size_t pqi_ref_get_global_size(uint d) { return d == 0 ? tl_gsize : 1; }
size_t pqi_ref_get_local_id(uint d) { return d == 0 ? tl_lid : 0; }
size_t pqi_ref_get_local_size(uint d) { return d == 0 ? tl_lsize : 1; }
size_t pqi_ref_get_group_id(uint d) { return d == 0 ? tl_grp : 0; }
void pqi_ref_barrier(int flags) {
  (void)flags;
  if (tl_lsize > 1) pthread_barrier_wait(tl_bar);
}

enum { K_CUT = 0, K_SINGLE = 1, K_DOUBLE = 2 };

typedef struct {
  int kind;
  const float* W;
  const void* theta;
  const int* args;
  float* max_e;
  int* max_i;
  float* loc_e;
  int* loc_i;
  size_t gid, lid, grp, gsize, lsize;
  pthread_barrier_t* bar;
} work_item;

static void* run_item(void* p) {
  work_item* it = (work_item*)p;
  tl_gid = it->gid;
  tl_lid = it->lid;
  tl_grp = it->grp;
  tl_gsize = it->gsize;
  tl_lsize = it->lsize;
  tl_bar = it->bar;
  switch (it->kind) {
    case K_CUT:
      calculate_cut(it->W, (uint*)it->theta, it->args, it->max_e, it->max_i, it->loc_e, it->loc_i);
      break;
    case K_SINGLE:
      single_bit_flips(it->W, (const uint*)it->theta, it->args, it->max_e, it->max_i, it->loc_e,
                       it->loc_i);
      break;
    default:
      double_bit_flips(it->W, (const uint*)it->theta, it->args, it->max_e, it->max_i, it->loc_e,
                       it->loc_i);
      break;
  }
  return NULL;
}

/* Launch one of the argmax-reducing kernels on a 1-D ND-range (G, L). */
static int launch_reducing(int kind, const float* W, const void* theta, const int* args, int G,
                           int L, float* max_e, int* max_i) {
  if (G <= 0 || L <= 0 || L > 1024 || G % L) return -1;
  const int groups = G / L;
  const int wave = L >= 256 ? 1 : 256 / L;  /* groups running at once */
  work_item* items = (work_item*)calloc((size_t)wave * L, sizeof(work_item));
  pthread_t* th = (pthread_t*)calloc((size_t)wave * L, sizeof(pthread_t));
  float* loc_e = (float*)calloc((size_t)wave * L, sizeof(float));
  int* loc_i = (int*)calloc((size_t)wave * L, sizeof(int));
  pthread_barrier_t* bars = (pthread_barrier_t*)calloc((size_t)wave, sizeof(pthread_barrier_t));
  if (!items || !th || !loc_e || !loc_i || !bars) return -2;
  pthread_attr_t attr;
  pthread_attr_init(&attr);
  pthread_attr_setstacksize(&attr, 1 << 20);
  for (int g0 = 0; g0 < groups; g0 += wave) {
    const int gn = groups - g0 < wave ? groups - g0 : wave;
    for (int q = 0; q < gn; ++q) pthread_barrier_init(&bars[q], NULL, (unsigned)L);
    for (int q = 0; q < gn; ++q) {
      const int g = g0 + q;
      for (int l = 0; l < L; ++l) {
        work_item* it = &items[(size_t)q * L + l];
        it->kind = kind;
        it->W = W;
        it->theta = theta;
        it->args = args;
        it->max_e = max_e;
        it->max_i = max_i;
        it->loc_e = loc_e + (size_t)q * L;
        it->loc_i = loc_i + (size_t)q * L;
        it->gid = (size_t)g * L + l;
        it->lid = (size_t)l;
        it->grp = (size_t)g;
        it->gsize = (size_t)G;
        it->lsize = (size_t)L;
        it->bar = &bars[q];
        if (L == 1 && gn == 1) {
          run_item(it);
        } else {
          pthread_create(&th[(size_t)q * L + l], &attr, run_item, it);
        }
      }
    }
    if (L > 1 || gn > 1)
      for (int t = 0; t < gn * L; ++t) pthread_join(th[t], NULL);
    for (int q = 0; q < gn; ++q) pthread_barrier_destroy(&bars[q]);
  }
  pthread_attr_destroy(&attr);
  free(items);
  free(th);
  free(loc_e);
  free(loc_i);
  free(bars);
  return 0;
}

int pqi_ref_calculate_cut(const float* W, int n, uint32_t* theta, int shots, int is_spin_glass,
                          int G, int L, float* max_e, int* max_i) {
  int args[5] = {n, shots, is_spin_glass, 0, 0};
  return launch_reducing(K_CUT, W, theta, args, G, L, max_e, max_i);
}

int pqi_ref_single_bit_flips(const float* W, int n, const uint32_t* theta, int is_spin_glass,
                             int G, int L, float* max_e, int* max_i) {
  int args[3] = {n, is_spin_glass, 0};
  return launch_reducing(K_SINGLE, W, theta, args, G, L, max_e, max_i);
}

int pqi_ref_double_bit_flips(const float* W, int n, const uint32_t* theta, int is_spin_glass,
                             int G, int L, float* max_e, int* max_i) {
  int args[3] = {n, is_spin_glass, 0};
  return launch_reducing(K_DOUBLE, W, theta, args, G, L, max_e, max_i);
}

/* gray has no barrier: each work-item runs on its own (local size 1). */
int pqi_ref_gray(const float* W, int n, const uint64_t* theta, int is_spin_glass, int iters_bound,
                 int G, uint64_t* theta_out, float* energy_out) {
  int args[4] = {n, is_spin_glass, iters_bound, 0};
  for (int g = 0; g < G; ++g) {
    tl_gid = (size_t)g;
    tl_lid = 0;
    tl_grp = (size_t)g;
    tl_gsize = (size_t)G;
    tl_lsize = 1;
    tl_bar = NULL;
    gray(W, (const ulong*)theta, args, (ulong*)theta_out, energy_out);
  }
  return 0;
}
